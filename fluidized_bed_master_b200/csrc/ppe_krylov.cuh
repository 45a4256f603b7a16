// ppe_krylov.cuh -- the pressure Poisson equation solved to a relative
// residual (engine extension; the reference does one Jacobi sweep,
// functions_PPE2.cuh:542-698, 868-878).
//
// The operator is the reference's: for a fluid particle i (the rows the
// reference's sweep updates)
//     d_i p_i - sum_j a_ij p_j = b_i,    d_i = sum_j a_ij,
//     a_ij = m_j (eps_i rho_i + eps_j rho_j) / (rho_i rho_j) * (-r.L grad W)/r^2,
// so one Jacobi sweep from the previous pressure is exactly the reference
// update.  Neighbours that are not solved for (walls, buffers) keep their
// current pressure and move to the right-hand side.  The coefficients are
// assembled once per step into a column-major array beside the neighbour
// list; every iteration then streams them (an HBM-bound pass) instead of
// recomputing the pair geometry.
//
// Solvers (Jacobi preconditioner M = diag(d)):
//   KRYLOV: right-preconditioned BiCGStab (the operator is not symmetric
//           once the gradient correction or unequal masses enter a_ij);
//   PCG:    preconditioned conjugate gradients in the Chronopoulos-Gear
//           form, whose three dot products all follow the one
//           matrix-vector product, so an iteration is two kernels: the
//           vector update and the product with its dots.
//           a_ij = m_j s_ij with s_ij symmetric (no gradient correction,
//           one smoothing length), so A is not symmetric when the masses
//           differ (they follow the porosity), but M A (M = diag(m)) is
//           symmetric positive definite.  CG runs on M A p = M b with the
//           preconditioner diag(M A) = M D, which is the same iteration on
//           A with every inner product weighted by m_i.
// Krylov vectors, dot products and norms are FP64; coefficients are R.
// Coefficient storage: entry k of row i = {j, a_ij} (8 B in the FP32
// build), solved neighbours only, in slices of 32 rows: the entries of
// rows 32s..32s+31 are one contiguous block, entry k of the slice's rows
// adjacent (kent_at), so a warp's load of entry k is one 256-B line pair
// and a warp's whole row block one contiguous stream.
// Dot products are reduced deterministically: every block writes a
// partial sum; the kernel that needs the totals (or the last block of the
// producing kernel) adds the partials in block order.
// The iteration runs inside the step's CUDA graph as a conditional while
// node; the last kernel of an iteration decides whether to continue.
#pragma once
#include <cuda_bf16.h>
#include "../../include/sphdem.h"
#include "step_kernels.cuh"

namespace sphdem {

constexpr int KRY_G = 1184;  // blocks of the vector kernels (8 per SM)
constexpr int KRY_GS = 444;  // blocks of the CG product: the 3 per SM its registers allow, one wave
constexpr int KRY_T = 256;
constexpr int KRY_NPART = 10;

// scalar slots
enum {
    KS_RHO = 0, KS_RHO_NEW, KS_ALPHA, KS_OMEGA, KS_BNORM, KS_RES, KS_DONE, KS_ITER, KS_RZ, KS_RZ_NEW,
    KS_TOL, KS_MAXIT, KS_STATUS, KS_RES0, KS_C0, KS_C1, KS_C2, KS_BETA, KS_COUNT = 24
};
// partial-sum slots
enum { KP_RHR = 0, KP_RR, KP_RHV, KP_SS, KP_TS, KP_TT, KP_BB, KP_PQ };

// one stored coefficient: {neighbour slot, a_ij}
template <typename R>
struct KEnt;
template <>
struct KEnt<float> {
    using T = int2;
    static __device__ __forceinline__ T make(int j, float a) { return make_int2(j, __float_as_int(a)); }
    static __device__ __forceinline__ void get(const T& e, int& j, double& a) {
        j = e.x;
        a = (double)__int_as_float(e.y);
    }
};
template <>
struct KEnt<double> {
    using T = int4;
    static __device__ __forceinline__ T make(int j, double a) {
        return make_int4(j, 0, __double2loint(a), __double2hiint(a));
    }
    static __device__ __forceinline__ void get(const T& e, int& j, double& a) {
        j = e.x;
        a = __hiloint2double(e.w, e.z);
    }
};

// slot of entry k of row i (cap entries per row)
__device__ __forceinline__ size_t kent_at(int i, int k, int cap) {
    return ((size_t)(i >> 5) * cap + k) * 32 + (i & 31);
}

template <typename R>
struct KryWork {
    typename KEnt<R>::T* e;   // entries of the solved neighbours, slot kent_at(i, k, cap)
    int cap;                  // entries per row
    int* kcnt;     // 0 for rows that are not solved, else 1 + the row's entries
    unsigned* ctr; // blocks finished in the current k_cg_spmv (the last one resets it)
    double* wm;    // m_i of solved rows (0 elsewhere): the weight of the PCG inner products
    double *d, *b, *x, *r, *rh, *p, *v, *s, *t, *y, *z;
    double* part;  // KRY_NPART * KRY_G block partials
    double* sc;    // KS_COUNT scalars
    // learned warm start (nullptr when it is off)
    float* fraw;           // [n][16] raw features (0 on rows that are not solved)
    __nv_bfloat16* feat;   // [n][16] normalised features, the network's input
    double* pprev;         // previous pressure of every row
    double* x0;            // the projected initial iterate of the solve (training target base)
    float *yp, *target, *weight;
    double* mpart;         // block partials of the feature statistics (33 per block)
    double* mstat;         // mean[16] | var[16] | pressure scale | rows | samples seen | Adam step
    // projected warm start (nullptr when it is off)
    float* D;              // [n][PROJ_MP] directions
    float* hist;           // [SPHDEM_WARM_HIST_MAX][hist_n] solution changes by particle id
    int hist_n;
    int* hring;            // {next slot, changes stored}
    double* ppart;         // PROJ_NV * KRY_G block partials
    double* pc;            // PROJ_MAX coefficients, directions kept, c.h
    double* AD;            // [PROJ_MAX][n] products A d_q of the last fit
};

// learned warm start statistics slots
enum { MS_MEAN = 0, MS_VAR = 16, MS_PS = 32, MS_ROWS = 33, MS_SEEN = 34, MS_T = 35, MS_COUNT = 40 };
constexpr int MLP_FEAT = 16;
constexpr int MPART_W = 2 * MLP_FEAT + 2;   // sum f | sum f^2 | rows | sum dp^2

// ---- reductions ----------------------------------------------------------
__device__ __forceinline__ double block_sum(double v, double* sm) {
    v = warp_sum(v);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sm[w] = v;
    __syncthreads();
    double t = 0;
    if (w == 0) {
        t = (l < (int)(blockDim.x >> 5)) ? sm[l] : 0.0;
        t = warp_sum(t);
        if (l == 0) sm[0] = t;
    }
    __syncthreads();
    t = sm[0];
    __syncthreads();
    return t;
}
// total of one partial slot, the same value in every block
__device__ __forceinline__ double part_total(const double* part, int slot, double* sm) {
    double v = 0;
    for (int k = threadIdx.x; k < KRY_G; k += blockDim.x) v += part[slot * KRY_G + k];
    return block_sum(v, sm);
}
__device__ __forceinline__ void part_store(double* part, int slot, double v, double* sm) {
    double t = block_sum(v, sm);
    if (threadIdx.x == 0) part[slot * KRY_G + blockIdx.x] = t;
}

__device__ __forceinline__ bool kry_solve_row(const DevParams& P, int it, int pt, int bt) {
    return it <= 2 && !(P.open_bc > 0 && bt > 0) && pt < 1000 && pt > 0;
}

// ---- assembly: coefficients, diagonal, right-hand side, initial iterate --
// Same neighbour terms and source as k_ppe.  Initial iterate: the previous
// pressure, plus its last change when extrapolate is set (the learned
// warm start overwrites it later).
template <typename R>
__global__ void __launch_bounds__(128) k_kry_assemble(DevParams P, SphState<R> S, SphWork<R> W, KryWork<R> K,
                                                      int extrapolate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    const SphRec<R> rec = W.rec;
    int it = S.itype[i], pt = S.ptype[i], bt = S.btype[i];
    V4<R> upi = rec.up[i];
    if (!kry_solve_row(P, it, pt, bt)) {
        K.kcnt[i] = 0;
        K.wm[i] = 0.0;
        K.d[i] = 1.0;
        K.b[i] = 0.0;
        K.x[i] = 0.0;
        if (K.fraw) {
            float* f = K.fraw + (size_t)i * MLP_FEAT;
#pragma unroll
            for (int q = 0; q < MLP_FEAT; q++) f[q] = 0.f;
            K.pprev[i] = (double)upi.w;
        }
        return;
    }
    R th = (R)S.h[i];
    Knl<R> Kn = knl_make<R>(P, th);
    PosRec<R> qi = ldr(rec.pos + i);
    V4<R> fi = rec.f1[i];
    R uxi = upi.x, uyi = upi.y, uzi = upi.z, rhoi = fi.y, pori = fi.w;
    R irhoi = rcp(rhoi), prhoi = pori * rhoi;
    R pux = pori * uxi, puy = pori * uyi, puz = pori * uzi;
    const bool kgc = P.kgc == 1;
    Cm9<R> Cm = cm_load(W.Cm, n, i, kgc);
    int cnt = min(W.ncnt[i], P.nb_cap);
    R bx = 0, by = 0, bz = 0;
    double dsum = 0, bfix = 0;
    // learned warm start: sum a_ij p_j over all neighbours, neighbour pressures
    double apsum = 0, pmean = 0, pmin = 1e300, pmax = -1e300;
    int np = 0;
    const int* __restrict__ nb = W.nbr;
    int k = 0;
    typename KEnt<R>::T* __restrict__ ent = K.e;
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
            if (!(tag_ptype(tj) >= 1000 || tag_itype(tj) == 4)) {
                const V4<R>& fj = t.a;
                const V4<R>& uj = t.b;
                Disp<R> g = disp(P, qi, t.q, S.x, S.y, S.z, i, j);
                R r2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz, r, rinv;
                rdist(r2, r, rinv);
                R mj = fj.x, rhoj = fj.y, porj = fj.w, irj = rcp(rhoj);
                R dw = kdw(Kn, r);
                R gx = dw * g.dx * rinv, gy = dw * g.dy * rinv, gz = dw * g.dz * rinv;
                cm_apply(Cm, kgc, gx, gy, gz);
                R mr = mj * irj;
                bx += mr * (pux - porj * uj.x) * gx;
                by += mr * (puy - porj * uj.y) * gy;
                bz += mr * (puz - porj * uj.z) * gz;
                R c = -(g.dx * gx + g.dy * gy + g.dz * gz) * rinv * rinv;
                R a = mj * ((prhoi + porj * rhoj) * irj * irhoi) * c;
                dsum += (double)a;
                if (kry_solve_row(P, tag_itype(tj), tag_ptype(tj), tag_btype(tj))) {
                    ent[kent_at(i, k, K.cap)] = KEnt<R>::make(j, a);
                    k++;
                } else {
                    bfix += (double)a * (double)uj.w;
                }
                double pj = (double)uj.w;
                apsum += (double)a * pj;
                pmean += pj;
                pmin = fmin(pmin, pj);
                pmax = fmax(pmax, pj);
                np++;
            }
        });
    R bdiv = (R)P.rho_gas * (bx + by + bz) / (R)P.sdt;
    R bpor = (R)P.rho_gas * ((R)2 * S.dDEMpor[i] - W.dDEMpor_prev[i]) / (R)P.sdt;
    R bsrc = (R)P.rho_gas * (bx + by + bz + (R)2 * S.dDEMpor[i] - W.dDEMpor_prev[i]) / (R)P.sdt;
    K.kcnt[i] = k + 1;
    K.wm[i] = (double)fi.x;
    K.d[i] = dsum;
    K.b[i] = (double)bsrc + bfix;
    K.x[i] = (double)upi.w + (extrapolate ? (double)S.dpres[i] : 0.0);
    if (K.fraw) {
        // features of the learned warm start: the previous pressure, the
        // reference's one-sweep update (b_i + sum_j a_ij p_j)/d_i and its
        // increment, neighbour pressure statistics, the terms of the
        // right-hand side, density deviation, porosity, neighbour count,
        // height, the pressure change of the previous solve, wall coupling
        // and the diagonal's magnitude
        double pi = (double)upi.w, idg = dsum > 0 ? 1.0 / dsum : 0.0;
        double jac = dsum > 0 ? ((double)bsrc + apsum) * idg : pi;
        pmean = np ? pmean / np : pi;
        if (np == 0) pmin = pmax = pi;
        float* f = K.fraw + (size_t)i * MLP_FEAT;
        f[0] = (float)pi;
        f[1] = (float)jac;
        f[2] = (float)(jac - pi);
        f[3] = (float)(pmean - pi);
        f[4] = (float)(pmin - pi);
        f[5] = (float)(pmax - pi);
        f[6] = (float)((double)bsrc * idg);
        f[7] = (float)((double)bdiv * idg);
        f[8] = (float)((fi.y - W.rho_ref[i]) / W.rho_ref[i]);
        f[9] = (float)pori;
        f[10] = (float)cnt;
        f[11] = (float)((double)bpor * idg);
        f[12] = (float)S.z[i];
        f[13] = (float)S.dpres[i];   // pressure change of the previous solve
        f[14] = (float)(bfix * idg);
        f[15] = (float)log10(fmax(dsum, 1e-30));
        K.pprev[i] = pi;
    }
}

// y_i = d_i x_i - sum_k a_ik x_j(k) over the stored entries of row i, in
// list order.  Software pipelined: the entries of the next group of B load
// while the current group's gathers are in flight (B = 8 measured best:
// 57 us per PCG iteration on the bench bed against 72 us unpipelined).
template <typename R, int B = 8>
__device__ __forceinline__ double kry_row(const KryWork<R>& K, int n, int i, int cnt, const double* __restrict__ xin) {
    using E = KEnt<R>;
    using T = typename E::T;
    const T* __restrict__ ent = K.e + kent_at(i, 0, K.cap);   // entry k at ent[32 k]
    (void)n;
    T cur[B], nxt[B];
#pragma unroll
    for (int q = 0; q < B; q++)
        if (q < cnt) cur[q] = __ldg(ent + (size_t)q * 32);
    double acc = 0;
    for (int k = 0; k < cnt; k += B) {
#pragma unroll
        for (int q = 0; q < B; q++)
            if (k + B + q < cnt) nxt[q] = __ldg(ent + (size_t)(k + B + q) * 32);
        double xv[B], av[B];
#pragma unroll
        for (int q = 0; q < B; q++) {
            xv[q] = 0.0;
            av[q] = 0.0;
            if (k + q < cnt) {
                int j;
                E::get(cur[q], j, av[q]);
                xv[q] = __ldg(xin + j);
            }
        }
#pragma unroll
        for (int q = 0; q < B; q++)
            if (k + q < cnt) acc += av[q] * xv[q];
#pragma unroll
        for (int q = 0; q < B; q++) cur[q] = nxt[q];
    }
    return K.d[i] * xin[i] - acc;
}

// y = A x over the stored coefficients; optional fused dots
// part[s0] += w0.y, part[s1] += w1.y (w1 == nullptr: y.y)
template <typename R>
__global__ void __launch_bounds__(KRY_T) k_kry_spmv(int n, KryWork<R> K, const int* __restrict__ nb,
                                                    const double* __restrict__ xin, double* __restrict__ yout,
                                                    const double* __restrict__ w0, int s0, const double* w1, int s1,
                                                    int two) {
    __shared__ double sm[32];
    (void)nb;
    if (K.sc[KS_DONE] != 0.0) return;
    double d0 = 0, d1 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int cnt = K.kcnt[i];
        double y = cnt ? kry_row<R>(K, n, i, cnt - 1, xin) : 0.0;
        yout[i] = y;
        d0 += w0[i] * y;
        if (two) d1 += (w1 ? w1[i] : y) * y;
    }
    part_store(K.part, s0, d0, sm);
    if (two) part_store(K.part, s1, d1, sm);
}

// r = b - y, rh = r, p = v = 0; part: rh.r, r.r, b.b   (BiCGStab)
// r = b - y, z = r/d, p = z;    part: r.z, r.r, b.b    (PCG)
__global__ void __launch_bounds__(KRY_T) k_kry_init(int n, double* __restrict__ d, const double* __restrict__ b,
                                                    const double* __restrict__ y, double* r, double* rh, double* p,
                                                    double* v, double* z, double* part, int cg) {
    __shared__ double sm[32];
    double a0 = 0, a1 = 0, a2 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ri = b[i] - y[i];
        r[i] = ri;
        if (cg) {
            double zi = ri / d[i];
            z[i] = zi;
            p[i] = zi;
            a0 += ri * zi;
        } else {
            rh[i] = ri;
            p[i] = 0.0;
            v[i] = 0.0;
            a0 += ri * ri;
        }
        a1 += ri * ri;
        a2 += b[i] * b[i];
    }
    part_store(part, KP_RHR, a0, sm);
    part_store(part, KP_RR, a1, sm);
    part_store(part, KP_BB, a2, sm);
}

// one block: initial scalars and the convergence state
__global__ void __launch_bounds__(KRY_T) k_kry_init_scalars(double* part, double* sc, double tol, int maxit, int cg) {
    __shared__ double sm[32];
    double rhr = part_total(part, KP_RHR, sm);
    double rr = part_total(part, KP_RR, sm);
    double bb = part_total(part, KP_BB, sm);
    if (threadIdx.x != 0) return;
    double bn = sqrt(bb);
    sc[KS_BNORM] = bn;
    sc[KS_TOL] = tol;
    sc[KS_MAXIT] = (double)maxit;
    sc[KS_ITER] = 0;
    sc[KS_STATUS] = 0;
    sc[KS_RHO] = 1.0;
    sc[KS_ALPHA] = 1.0;
    sc[KS_OMEGA] = 1.0;
    sc[KS_RZ] = rhr;
    double res = bn > 0 ? sqrt(rr) / bn : 0.0;
    sc[KS_RES] = res;
    sc[KS_RES0] = res;
    sc[KS_DONE] = (bn == 0.0 || res <= tol || maxit <= 0) ? 1.0 : 0.0;
    (void)cg;
}

// ---- BiCGStab iteration -------------------------------------------------
// B1: rho' = rh.r; beta = (rho'/rho)(alpha/omega); p = r + beta (p - omega v); y = p/d
__global__ void __launch_bounds__(KRY_T) k_bicg_p(int n, const double* __restrict__ d, const double* __restrict__ r,
                                                  double* p, const double* __restrict__ v, double* y, double* part,
                                                  double* sc) {
    __shared__ double sm[32];
    if (sc[KS_DONE] != 0.0) return;
    double rho_new = part_total(part, KP_RHR, sm);
    double beta = (rho_new / sc[KS_RHO]) * (sc[KS_ALPHA] / sc[KS_OMEGA]);
    double om = sc[KS_OMEGA];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double pi = r[i] + beta * (p[i] - om * v[i]);
        p[i] = pi;
        y[i] = pi / d[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) sc[KS_RHO_NEW] = rho_new;
}

// B3: alpha = rho'/(rh.v); s = r - alpha v; x += alpha y; z = s/d
__global__ void __launch_bounds__(KRY_T) k_bicg_s(int n, const double* __restrict__ d, const double* __restrict__ r,
                                                  const double* __restrict__ v, const double* __restrict__ y, double* x,
                                                  double* s, double* z, double* part, double* sc) {
    __shared__ double sm[32];
    if (sc[KS_DONE] != 0.0) return;
    double rv = part_total(part, KP_RHV, sm);
    if (!(rv != 0.0) || !isfinite(rv)) {   // breakdown: every block sees the same rv
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            sc[KS_DONE] = 1.0;
            sc[KS_STATUS] = 2.0;
        }
        return;
    }
    double alpha = sc[KS_RHO_NEW] / rv;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double si = r[i] - alpha * v[i];
        s[i] = si;
        x[i] += alpha * y[i];
        z[i] = si / d[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) sc[KS_ALPHA] = alpha;
}

// B5: omega = (t.s)/(t.t); x += omega z; r = s - omega t; part: rh.r, r.r
__global__ void __launch_bounds__(KRY_T) k_bicg_x(int n, const double* __restrict__ s, const double* __restrict__ t,
                                                  const double* __restrict__ z, const double* __restrict__ rh, double* x,
                                                  double* r, double* part, double* sc) {
    __shared__ double sm[32];
    if (sc[KS_DONE] != 0.0) return;
    double ts = part_total(part, KP_TS, sm);
    double tt = part_total(part, KP_TT, sm);
    double om = (tt > 0.0) ? ts / tt : 0.0;
    double a0 = 0, a1 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] += om * z[i];
        double ri = s[i] - om * t[i];
        r[i] = ri;
        a0 += rh[i] * ri;
        a1 += ri * ri;
    }
    part_store(part, KP_RHR, a0, sm);
    part_store(part, KP_RR, a1, sm);
    if (blockIdx.x == 0 && threadIdx.x == 0) sc[KS_OMEGA] = om;
}

// ---- PCG iteration (Chronopoulos-Gear) ----------------------------------
// With u = M^-1 r and w = A u, one iteration is
//     p = u + beta p;  s = w + beta s;  x += alpha p;  r -= alpha s;
//     u = M^-1 r;  w = A u;  gamma = r.u, delta = w.u, rho = r.r;
//     beta' = gamma/gamma_old;  alpha' = gamma / (delta - beta' gamma/alpha)
// (alpha = gamma/delta, beta = 0 at the start).  The iterates equal those
// of the textbook recurrences in exact arithmetic.
enum { KP_G = 0, KP_D = 1, KP_R = 2, KP_B = 3 };

// r = b - y, u = r/d, p = s = 0; the tolerance and the iteration cap
__global__ void __launch_bounds__(KRY_T) k_cg_init(int n, const double* __restrict__ d, const double* __restrict__ b,
                                                   const double* __restrict__ y, double* r, double* u, double* p,
                                                   double* s, double* sc, double tol, int maxit) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc[KS_TOL] = tol;
        sc[KS_MAXIT] = (double)maxit;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ri = b[i] - y[i];
        r[i] = ri;
        u[i] = ri / d[i];
        p[i] = 0.0;
        s[i] = 0.0;
    }
}

// p = u + beta p; s = w + beta s; x += alpha p; r -= alpha s; u = r/d
__global__ void __launch_bounds__(KRY_T) k_cg_upd(int n, const double* __restrict__ d, double* u,
                                                  const double* __restrict__ w, double* p, double* s, double* x,
                                                  double* r, const double* sc) {
    if (sc[KS_DONE] != 0.0) return;
    const double al = sc[KS_ALPHA], be = sc[KS_BETA];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double pi = u[i] + be * p[i];
        double si = w[i] + be * s[i];
        p[i] = pi;
        s[i] = si;
        x[i] += al * pi;
        double ri = r[i] - al * si;
        r[i] = ri;
        u[i] = ri / d[i];
    }
}

// w = A u with the partials of the m-weighted r.u and w.u, and of r.r
// (and b.b on the first call);
// the last block to finish adds the partials in block order and advances
// the scalars: the residual, the stop decision (and the while node's
// condition), alpha and beta of the next update
template <typename R>
__global__ void __launch_bounds__(KRY_T) k_cg_spmv(int n, KryWork<R> K, const double* __restrict__ u,
                                                   double* __restrict__ w, const double* __restrict__ r,
                                                   const double* __restrict__ b, int first,
                                                   cudaGraphConditionalHandle h, int in_graph) {
    __shared__ double sm[32];
    __shared__ int last;
    double* sc = K.sc;
    if (sc[KS_DONE] != 0.0) {
        if (in_graph && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
        return;
    }
    double g = 0, dl = 0, rr = 0, bb = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int cnt = K.kcnt[i];
        double ui = u[i];
        double wi = cnt ? kry_row<R>(K, n, i, cnt - 1, u) : 0.0;
        w[i] = wi;
        double ri = r[i], mi = K.wm[i];
        g += mi * ri * ui;
        dl += mi * wi * ui;
        rr += ri * ri;
        if (first) bb += b[i] * b[i];
    }
    part_store(K.part, KP_G, g, sm);
    part_store(K.part, KP_D, dl, sm);
    part_store(K.part, KP_R, rr, sm);
    if (first) part_store(K.part, KP_B, bb, sm);
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(K.ctr, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // totals in block order (the partials bypass L1: other SMs wrote them)
    double tot[4];
    for (int q = 0; q < (first ? 4 : 3); q++) {
        double v = 0;
        for (int k = threadIdx.x; k < gridDim.x; k += blockDim.x) v += __ldcg(K.part + q * KRY_G + k);
        tot[q] = block_sum(v, sm);
    }
    if (threadIdx.x != 0) return;
    *K.ctr = 0u;
    const double gam = tot[KP_G], del = tot[KP_D], rho = tot[KP_R];
    bool done;
    if (first) {
        double bn = sqrt(tot[KP_B]);
        sc[KS_BNORM] = bn;
        sc[KS_ITER] = 0;
        sc[KS_STATUS] = 0;
        double res = bn > 0 ? sqrt(rho) / bn : 0.0;
        sc[KS_RES] = res;
        sc[KS_RES0] = res;
        done = bn == 0.0 || res <= sc[KS_TOL] || sc[KS_MAXIT] <= 0;
        if (!done && (!(del != 0.0) || !isfinite(del))) {
            sc[KS_STATUS] = 2.0;
            done = true;
        }
        if (!done) {
            sc[KS_ALPHA] = gam / del;
            sc[KS_BETA] = 0.0;
            sc[KS_RZ] = gam;
        }
    } else {
        double it = sc[KS_ITER] + 1.0;
        sc[KS_ITER] = it;
        double res = sqrt(rho) / sc[KS_BNORM];
        sc[KS_RES] = res;
        done = true;
        if (!isfinite(res)) sc[KS_STATUS] = 2.0;
        else if (res <= sc[KS_TOL]) {
        } else if (it >= sc[KS_MAXIT]) sc[KS_STATUS] = 1.0;   // iteration cap
        else {
            double be = gam / sc[KS_RZ];
            double den = del - be * gam / sc[KS_ALPHA];
            if (!(den != 0.0) || !isfinite(den)) sc[KS_STATUS] = 2.0;
            else {
                sc[KS_BETA] = be;
                sc[KS_ALPHA] = gam / den;
                sc[KS_RZ] = gam;
                done = false;
            }
        }
    }
    if (done) sc[KS_DONE] = 1.0;
    if (in_graph) cudaGraphSetConditional(h, done ? 0u : 1u);
}

// last kernel of an iteration (one block): residual, iteration count, and
// whether the while node runs another iteration
__global__ void __launch_bounds__(KRY_T) k_kry_check(double* part, double* sc, cudaGraphConditionalHandle h,
                                                     int in_graph, int cg) {
    __shared__ double sm[32];
    bool done = sc[KS_DONE] != 0.0;
    double rr = done ? 0.0 : part_total(part, KP_RR, sm);
    if (threadIdx.x != 0) return;
    if (!done) {
        double it = sc[KS_ITER] + 1.0;
        sc[KS_ITER] = it;
        double res = sqrt(rr) / sc[KS_BNORM];
        sc[KS_RES] = res;
        if (cg) sc[KS_RZ] = sc[KS_RZ_NEW];
        else sc[KS_RHO] = sc[KS_RHO_NEW];
        bool stop = res <= sc[KS_TOL] || it >= sc[KS_MAXIT] || !isfinite(res) || (!cg && sc[KS_OMEGA] == 0.0);
        if (!isfinite(res) || (!cg && sc[KS_OMEGA] == 0.0)) sc[KS_STATUS] = 2.0;
        else if (stop && res > sc[KS_TOL]) sc[KS_STATUS] = 1.0;   // iteration cap
        if (stop) {
            sc[KS_DONE] = 1.0;
            done = true;
        }
    }
    if (in_graph) cudaGraphSetConditional(h, done ? 0u : 1u);
}

// ---- learned warm start: statistics, normalisation, targets ---------------
// Block partials over the solved rows (kcnt > 0): mode 0 sums the raw
// features and their squares; mode 1 sums (x - x0)^2 of the solution.
template <typename R>
__global__ void __launch_bounds__(KRY_T) k_mlp_stats(int n, KryWork<R> K, int mode) {
    __shared__ double sm[32];
    double acc[MPART_W];
#pragma unroll
    for (int q = 0; q < MPART_W; q++) acc[q] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (K.kcnt[i] == 0) continue;
        acc[2 * MLP_FEAT] += 1.0;
        if (mode == 0) {
            const float* f = K.fraw + (size_t)i * MLP_FEAT;
#pragma unroll
            for (int q = 0; q < MLP_FEAT; q++) {
                double v = f[q];
                acc[q] += v;
                acc[MLP_FEAT + q] += v * v;
            }
        } else {
            double dp = K.x[i] - K.x0[i];
            acc[2 * MLP_FEAT + 1] += dp * dp;
        }
    }
    for (int q = 0; q < MPART_W; q++) {
        double t = block_sum(acc[q], sm);
        if (threadIdx.x == 0) K.mpart[(size_t)blockIdx.x * MPART_W + q] = t;
    }
}

// one block: totals in block order, then the running statistics.  Feature
// mean/variance and the pressure scale are exponential averages (0.9) over
// training steps; the first training step sets them.
template <typename R>
__global__ void __launch_bounds__(KRY_T) k_mlp_stats_final(int nblocks, KryWork<R> K, int mode) {
    __shared__ double tot[MPART_W];
    int q = threadIdx.x;
    if (q < MPART_W) {
        double t = 0;
        for (int b = 0; b < nblocks; b++) t += K.mpart[(size_t)b * MPART_W + q];
        tot[q] = t;
    }
    __syncthreads();
    double rows = tot[2 * MLP_FEAT];
    double* M = K.mstat;
    if (q == 0) M[MS_ROWS] = rows;
    if (rows <= 0) return;
    if (mode == 0 && q < MLP_FEAT) {
        double mu = tot[q] / rows, var = fmax(tot[MLP_FEAT + q] / rows - mu * mu, 0.0);
        bool first = M[MS_SEEN] == 0.0;
        M[MS_MEAN + q] = first ? mu : 0.9 * M[MS_MEAN + q] + 0.1 * mu;
        M[MS_VAR + q] = first ? var : 0.9 * M[MS_VAR + q] + 0.1 * var;
    }
    if (mode == 1 && q == 0) {
        double ps = sqrt(tot[2 * MLP_FEAT + 1] / rows);
        if (!(ps > 0)) ps = 1.0;
        M[MS_PS] = M[MS_SEEN] == 0.0 ? ps : 0.9 * M[MS_PS] + 0.1 * ps;
        M[MS_SEEN] += 1.0;
    }
}

// normalised BF16 features of every row (zero on rows that are not solved)
template <typename R>
__global__ void k_mlp_norm(int n, KryWork<R> K) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * MLP_FEAT) return;
    int i = q / MLP_FEAT, c = q - i * MLP_FEAT;
    float v = 0.f;
    if (K.kcnt[i] > 0) {
        double sd = sqrt(K.mstat[MS_VAR + c]);
        v = (float)((K.fraw[q] - K.mstat[MS_MEAN + c]) / (sd > 1e-30 ? sd : 1.0));
    }
    K.feat[q] = __float2bfloat16_rn(v);
}

// initial iterate from the network: p_prev + scale * y on solved rows
template <typename R>
__global__ void k_mlp_x0(int n, KryWork<R> K) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || K.kcnt[i] == 0) return;
    K.x[i] = K.pprev[i] + K.mstat[MS_PS] * (double)K.yp[i];
}

// training pairs: target = (x - x0) / scale, the part of the solution that
// the projection without the network missed; weight = 1 / rows on solved rows
template <typename R>
__global__ void k_mlp_targets(int n, KryWork<R> K) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool on = K.kcnt[i] > 0;
    double rows = K.mstat[MS_ROWS];
    K.target[i] = on ? (float)((K.x[i] - K.x0[i]) / K.mstat[MS_PS]) : 0.f;
    K.weight[i] = (on && rows > 0) ? (float)(1.0 / rows) : 0.f;
}

__global__ void k_mlp_tick(double* mstat) { mstat[MS_T] += 1.0; }

// ---- projected initial iterate (warm starts PROJECT and MLP) ---------------
// x0 = sum_q c_q d_q over the directions
//     d0 = the previous pressure (FP64), d1 = the network's predicted
//     change (MLP in use, else 0), d2.. = the last warm_hist solution
//     changes, newest first (FP32),
// with c from the Galerkin equations (D^T M A D) c = D^T M b (the optimal
// combination in the norm of the symmetric operator M A, never worse than
// d0 alone in that norm), or (warm_fit RESIDUAL) from the least-squares equations
// (AD)^T (AD) c = (AD)^T b.  With warm_fit AFFINE, c0 = 1 and the other
// directions are fitted to r0 = b - A d0.  Directions
// are FP32 rows of PROJ_MP floats (one 48-B gather per list entry for all
// of them) except d0, gathered as FP64; their products with A and the dots
// are FP64.  The products are kept, so A x0 = sum_q c_q (A d_q) comes with
// x0 and the solver needs no product of its own before its first step.
// Directions that are zero or dependent are dropped from the system.
constexpr int PROJ_MAX = 2 + SPHDEM_WARM_HIST_MAX;   // 10
constexpr int PROJ_MP = 12;                          // floats per direction row
constexpr int PROJ_NG = PROJ_MAX * (PROJ_MAX + 1) / 2;
constexpr int PROJ_NV = PROJ_NG + PROJ_MAX;          // upper triangle of G, then h

template <typename R>
__global__ void k_proj_dirs(int n, KryWork<R> K, const int* __restrict__ pid, int nhist, int use_mlp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool on = K.kcnt[i] > 0;
    float d[PROJ_MP];
#pragma unroll
    for (int q = 0; q < PROJ_MP; q++) d[q] = 0.f;
    if (on) {
        // d[0] stays 0: the previous pressure enters the products as FP64
        if (use_mlp) d[1] = (float)(K.mstat[MS_PS] * (double)K.yp[i]);
        const int slot = K.hring[0], have = min(K.hring[1], nhist), p = pid[i];
        for (int k = 0; k < have; k++) {
            int s = (slot - 1 - k + SPHDEM_WARM_HIST_MAX) % SPHDEM_WARM_HIST_MAX;
            d[2 + k] = K.hist[(size_t)s * K.hist_n + p];
        }
    }
    float4* o = reinterpret_cast<float4*>(K.D + (size_t)i * PROJ_MP);
#pragma unroll
    for (int q = 0; q < PROJ_MP / 4; q++) o[q] = make_float4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
}

// (A d_q)_i for every direction in one pass over the stored coefficients,
// and the block partials of G (upper triangle) and h.  Each thread stages
// its row's products in shared memory; then thread v < PROJ_NV forms value
// v over the block's rows in row order: deterministic, no shuffles.
// G = the float4 groups of D that can be non-zero (slots 0..4G-1): with
// fewer history directions the pass gathers fewer direction bytes per
// neighbour; the slots above are zero, so their products are zero anyway.
constexpr int PROJ_T = 128;
__host__ __device__ constexpr int proj_groups(int nhist) { return (1 + nhist) / 4 + 1 < 3 ? (1 + nhist) / 4 + 1 : 3; }
template <typename R, int G = 3>
__global__ void __launch_bounds__(PROJ_T) k_proj_spmv(int n, KryWork<R> K, int fit) {
    using E = KEnt<R>;
    const bool least_squares = fit & SPHDEM_FIT_RESIDUAL, affine = fit & SPHDEM_FIT_AFFINE;
    __shared__ double su[PROJ_T][PROJ_MAX + 1];   // left factors (+ b or r0)
    __shared__ double sa[PROJ_T][PROJ_MAX];       // A d_q
    const float4* __restrict__ D4 = reinterpret_cast<const float4*>(K.D);
    const typename E::T* __restrict__ ent = K.e;
    double accv = 0.0;   // value threadIdx.x of this block
    int vk = 0, vq = 0;  // (k, q) of an upper-triangle value
    if (threadIdx.x < PROJ_NG) {
        int v = threadIdx.x;
        while (v >= PROJ_MAX - vk) { v -= PROJ_MAX - vk; vk++; }
        vq = vk + v;
    }
    for (int i0 = blockIdx.x * PROJ_T; i0 < n; i0 += gridDim.x * PROJ_T) {
        const int i = i0 + threadIdx.x;
        double ad[PROJ_MAX], dv[PROJ_MAX], bi = 0;
#pragma unroll
        for (int q = 0; q < PROJ_MAX; q++) ad[q] = dv[q] = 0.0;
        int cnt = i < n ? K.kcnt[i] : 0;
        if (cnt) {
            const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
            float4 a0 = D4[(size_t)i * 3], a1 = G > 1 ? D4[(size_t)i * 3 + 1] : z4,
                   a2 = G > 2 ? D4[(size_t)i * 3 + 2] : z4;
            float di[PROJ_MP] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w};
            const double dg = K.d[i];
#pragma unroll
            for (int q = 0; q < PROJ_MAX; q++) {
                dv[q] = q == 0 ? K.x[i] : (double)di[q];
                ad[q] = dg * dv[q];
            }
            const double* __restrict__ xp = K.x;   // d0 = the previous pressure, FP64
            // entries in pairs: both entries' direction gathers are in
            // flight before their updates
            const typename E::T* __restrict__ er = ent + kent_at(i, 0, K.cap);
            const int ne = cnt - 1;
            int k = 0;
            for (; k + 2 <= ne; k += 2) {
                int j0, j1;
                double a0, a1;
                E::get(__ldg(er + (size_t)k * 32), j0, a0);
                E::get(__ldg(er + (size_t)(k + 1) * 32), j1, a1);
                float4 p0 = __ldg(D4 + (size_t)j0 * 3), p1 = G > 1 ? __ldg(D4 + (size_t)j0 * 3 + 1) : z4,
                       p2 = G > 2 ? __ldg(D4 + (size_t)j0 * 3 + 2) : z4;
                float4 q0 = __ldg(D4 + (size_t)j1 * 3), q1 = G > 1 ? __ldg(D4 + (size_t)j1 * 3 + 1) : z4,
                       q2 = G > 2 ? __ldg(D4 + (size_t)j1 * 3 + 2) : z4;
                const double x0j = __ldg(xp + j0), x1j = __ldg(xp + j1);
                float d0[PROJ_MP] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w, p2.x, p2.y, p2.z, p2.w};
                float d1[PROJ_MP] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};
                ad[0] -= a0 * x0j;
#pragma unroll
                for (int q = 1; q < PROJ_MAX; q++) ad[q] -= a0 * (double)d0[q];
                ad[0] -= a1 * x1j;
#pragma unroll
                for (int q = 1; q < PROJ_MAX; q++) ad[q] -= a1 * (double)d1[q];
            }
            for (; k < ne; k++) {
                int j;
                double a;
                E::get(__ldg(er + (size_t)k * 32), j, a);
                float4 b0 = __ldg(D4 + (size_t)j * 3), b1 = G > 1 ? __ldg(D4 + (size_t)j * 3 + 1) : z4,
                       b2 = G > 2 ? __ldg(D4 + (size_t)j * 3 + 2) : z4;
                float dj[PROJ_MP] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w, b2.x, b2.y, b2.z, b2.w};
                ad[0] -= a * __ldg(xp + j);
#pragma unroll
                for (int q = 1; q < PROJ_MAX; q++) ad[q] -= a * (double)dj[q];
            }
        }
        // the products, for A x0 in k_proj_apply (0 on rows that are not solved)
        if (i < n) {
#pragma unroll
            for (int q = 0; q < PROJ_MAX; q++) K.AD[(size_t)q * n + i] = ad[q];
        }
        if (cnt) {
            bi = affine ? K.b[i] - ad[0] : K.b[i];   // ad[0] = (A p_prev)_i
            if (affine) dv[0] = ad[0] = 0.0;          // p_prev is not fitted
            // Galerkin: the m-weighted products (M A is the symmetric operator)
            if (!least_squares) {
                const double wgt = K.wm[i];
#pragma unroll
                for (int q = 0; q < PROJ_MAX; q++) dv[q] *= wgt;
            }
        }
#pragma unroll
        for (int q = 0; q < PROJ_MAX; q++) {
            su[threadIdx.x][q] = least_squares ? ad[q] : dv[q];
            sa[threadIdx.x][q] = ad[q];
        }
        su[threadIdx.x][PROJ_MAX] = bi;
        __syncthreads();
        if (threadIdx.x < PROJ_NG) {
            for (int r = 0; r < PROJ_T; r++) accv += su[r][vk] * sa[r][vq];
        } else if (threadIdx.x < PROJ_NV) {
            const int k = threadIdx.x - PROJ_NG;
            for (int r = 0; r < PROJ_T; r++) accv += su[r][k] * su[r][PROJ_MAX];
        }
        __syncthreads();
    }
    if (threadIdx.x < PROJ_NV) K.ppart[(size_t)threadIdx.x * KRY_G + blockIdx.x] = accv;
}

// one block: totals in block order (thread v adds value v), then the
// reduced system of the kept directions (Gaussian elimination with partial
// pivoting and a relative ridge of 1e-12 trace); c = e0 (the previous
// pressure) if it fails
template <typename R>
__global__ void __launch_bounds__(KRY_T) k_proj_solve(KryWork<R> K, int nblk) {
    __shared__ double tot[PROJ_NV];
    if (threadIdx.x < PROJ_NV) {
        const double* pv = K.ppart + (size_t)threadIdx.x * KRY_G;
        double t = 0;
        for (int k = 0; k < nblk; k++) t += pv[k];
        tot[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double G[PROJ_MAX][PROJ_MAX], h[PROJ_MAX], c[PROJ_MAX];
    int v = 0;
    for (int k = 0; k < PROJ_MAX; k++)
        for (int q = k; q < PROJ_MAX; q++, v++) G[k][q] = G[q][k] = tot[v];
    double gmax = 0;
    for (int k = 0; k < PROJ_MAX; k++) {
        h[k] = tot[PROJ_NG + k];
        c[k] = 0;
        gmax = fmax(gmax, fabs(G[k][k]));
    }
    // kept directions: a diagonal above 1e-14 of the largest
    int idx[PROJ_MAX], m = 0;
    for (int k = 0; k < PROJ_MAX; k++)
        if (G[k][k] > 1e-14 * gmax && isfinite(G[k][k])) idx[m++] = k;
    double M[PROJ_MAX][PROJ_MAX + 1];
    double tr = 0;
    for (int a = 0; a < m; a++) tr += G[idx[a]][idx[a]];
    for (int a = 0; a < m; a++) {
        for (int b = 0; b < m; b++) M[a][b] = G[idx[a]][idx[b]];
        M[a][a] += 1e-12 * tr;
        M[a][m] = h[idx[a]];
    }
    bool ok = m > 0 && tr > 0 && isfinite(tr);
    for (int k = 0; k < m && ok; k++) {
        int piv = k;
        for (int r = k + 1; r < m; r++)
            if (fabs(M[r][k]) > fabs(M[piv][k])) piv = r;
        if (!(fabs(M[piv][k]) > 0)) { ok = false; break; }
        for (int q = 0; q <= m; q++) { double t = M[k][q]; M[k][q] = M[piv][q]; M[piv][q] = t; }
        for (int r = k + 1; r < m; r++) {
            double f = M[r][k] / M[k][k];
            for (int q = k; q <= m; q++) M[r][q] -= f * M[k][q];
        }
    }
    double x[PROJ_MAX];
    if (ok) {
        for (int k = m - 1; k >= 0; k--) {
            double t = M[k][m];
            for (int q = k + 1; q < m; q++) t -= M[k][q] * x[q];
            x[k] = t / M[k][k];
            ok = ok && isfinite(x[k]);
        }
    }
    double gain = 0;
    if (ok)
        for (int a = 0; a < m; a++) {
            c[idx[a]] = x[a];
            gain += x[a] * h[idx[a]];
        }
    else c[0] = 1.0;   // (an affine fit keeps p_prev whatever c0 is)
    for (int k = 0; k < PROJ_MAX; k++) K.pc[k] = c[k];
    K.pc[PROJ_MAX] = ok ? m : 0;   // diagnostics: directions kept, c.h
    K.pc[PROJ_MAX + 1] = gain;
}

// x0 = c0 p_prev (FP64) + sum_{q>0} c_q d_q   (c0 = 1 for an affine fit)
// and y = A x0 = c0 (A p_prev) + sum_{q>0} c_q (A d_q) from the kept products
template <typename R>
__global__ void k_proj_apply(int n, KryWork<R> K, int fit) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (K.kcnt[i] == 0) {
        K.y[i] = 0.0;
        return;
    }
    const float* d = K.D + (size_t)i * PROJ_MP;
    const double c0 = (fit & SPHDEM_FIT_AFFINE) ? 1.0 : K.pc[0];
    double x = c0 * K.x[i], y = c0 * K.AD[i];
#pragma unroll
    for (int q = 1; q < PROJ_MAX; q++) {
        x += K.pc[q] * (double)d[q];
        y += K.pc[q] * K.AD[(size_t)q * n + i];
    }
    K.x[i] = x;
    K.y[i] = y;
    if (K.x0) K.x0[i] = x;
}

// advance the ring of solution changes after k_kry_final wrote the newest
__global__ void k_proj_ring(int* hring) {
    hring[0] = (hring[0] + 1) % SPHDEM_WARM_HIST_MAX;
    hring[1] = min(hring[1] + 1, SPHDEM_WARM_HIST_MAX);
}

// p_new = x on solved rows, the current pressure elsewhere; the change
// also goes into the ring of solution changes (by particle id) when the
// projected warm start keeps one
template <typename R>
__global__ void __launch_bounds__(128) k_kry_final(DevParams P, SphState<R> S, SphWork<R> W, KryWork<R> K) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.ns) return;
    bool solve = kry_solve_row(P, S.itype[i], S.ptype[i], S.btype[i]);
    R pold = W.rec.up[i].w;
    double dp = solve ? K.x[i] - (double)pold : 0.0;
    W.p_new[i] = solve ? (R)K.x[i] : pold;
    S.dpres[i] = (R)dp;
    if (K.hist) K.hist[(size_t)K.hring[0] * K.hist_n + S.pid[i]] = (float)dp;
}

}  // namespace sphdem
