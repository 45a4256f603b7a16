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
//   PCG:    preconditioned conjugate gradients (symmetric operators).
// Krylov vectors, dot products and norms are FP64; coefficients are R.
// Dot products are reduced deterministically: every block writes a
// partial sum, and the next kernel adds the partials in a fixed order.
// The iteration runs inside the step's CUDA graph as a conditional while
// node; the last kernel of an iteration decides whether to continue.
#pragma once
#include "step_kernels.cuh"

namespace sphdem {

constexpr int KRY_G = 592;   // blocks of the vector kernels (4 per SM)
constexpr int KRY_T = 256;
constexpr int KRY_NPART = 10;

// scalar slots
enum {
    KS_RHO = 0, KS_RHO_NEW, KS_ALPHA, KS_OMEGA, KS_BNORM, KS_RES, KS_DONE, KS_ITER, KS_RZ, KS_RZ_NEW,
    KS_TOL, KS_MAXIT, KS_STATUS, KS_RES0, KS_C0, KS_C1, KS_C2, KS_COUNT = 24
};
// partial-sum slots
enum { KP_RHR = 0, KP_RR, KP_RHV, KP_SS, KP_TS, KP_TT, KP_BB, KP_PQ };

template <typename R>
struct KryWork {
    R* a;          // cap*ns coefficients a[k*n+i] of list entry k (0: not a solved neighbour)
    int* kcnt;     // list entries a row uses (0 for rows that are not solved)
    double *d, *b, *x, *r, *rh, *p, *v, *s, *t, *y, *z;
    double* part;  // KRY_NPART * KRY_G block partials
    double* sc;    // KS_COUNT scalars
    // learned warm start (nullptr when it is off)
    float* fraw;           // [n][16] raw features (0 on rows that are not solved)
    __nv_bfloat16* feat;   // [n][16] normalised features, the network's input
    double* pprev;         // previous pressure of every row
    float *yp, *target, *weight;
    double* mpart;         // block partials of the feature statistics (33 per block)
    double* mstat;         // mean[16] | var[16] | pressure scale | rows | samples seen | Adam step
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
    nb_walk<2, NbQ44<R>>(
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
            R acoef = 0;
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
                if (kry_solve_row(P, tag_itype(tj), tag_ptype(tj), tag_btype(tj))) acoef = a;
                else bfix += (double)a * (double)uj.w;
                double pj = (double)uj.w;
                apsum += (double)a * pj;
                pmean += pj;
                pmin = fmin(pmin, pj);
                pmax = fmax(pmax, pj);
                np++;
            }
            K.a[(size_t)k * n + i] = acoef;
            k++;
        });
    R bdiv = (R)P.rho_gas * (bx + by + bz) / (R)P.sdt;
    R bpor = (R)P.rho_gas * ((R)2 * S.dDEMpor[i] - W.dDEMpor_prev[i]) / (R)P.sdt;
    R bsrc = (R)P.rho_gas * (bx + by + bz + (R)2 * S.dDEMpor[i] - W.dDEMpor_prev[i]) / (R)P.sdt;
    K.kcnt[i] = cnt;
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

// y = A x over the stored coefficients; optional fused dots
// part[s0] += w0.y, part[s1] += w1.y (w1 == nullptr: y.y)
template <typename R>
__global__ void __launch_bounds__(KRY_T) k_kry_spmv(int n, KryWork<R> K, const int* __restrict__ nb,
                                                    const double* __restrict__ xin, double* __restrict__ yout,
                                                    const double* __restrict__ w0, int s0, const double* w1, int s1,
                                                    int two) {
    __shared__ double sm[32];
    if (K.sc[KS_DONE] != 0.0) return;
    double d0 = 0, d1 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int cnt = K.kcnt[i];
        double acc = 0;
        int k = 0;
        for (; k + 4 <= cnt; k += 4) {
            int j0 = __ldg(nb + (size_t)k * n + i), j1 = __ldg(nb + (size_t)(k + 1) * n + i);
            int j2 = __ldg(nb + (size_t)(k + 2) * n + i), j3 = __ldg(nb + (size_t)(k + 3) * n + i);
            R a0 = __ldg(K.a + (size_t)k * n + i), a1 = __ldg(K.a + (size_t)(k + 1) * n + i);
            R a2 = __ldg(K.a + (size_t)(k + 2) * n + i), a3 = __ldg(K.a + (size_t)(k + 3) * n + i);
            acc += (double)a0 * xin[j0];
            acc += (double)a1 * xin[j1];
            acc += (double)a2 * xin[j2];
            acc += (double)a3 * xin[j3];
        }
        for (; k < cnt; k++) acc += (double)__ldg(K.a + (size_t)k * n + i) * xin[__ldg(nb + (size_t)k * n + i)];
        double y = cnt ? K.d[i] * xin[i] - acc : 0.0;
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

// ---- PCG iteration --------------------------------------------------------
// C2: alpha = rz/(p.q); x += alpha p; r -= alpha q; z = r/d; part: r.z, r.r
__global__ void __launch_bounds__(KRY_T) k_cg_x(int n, const double* __restrict__ d, const double* __restrict__ p,
                                                const double* __restrict__ q, double* x, double* r, double* z,
                                                double* part, double* sc) {
    __shared__ double sm[32];
    if (sc[KS_DONE] != 0.0) return;
    double pq = part_total(part, KP_PQ, sm);
    if (!(pq != 0.0) || !isfinite(pq)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            sc[KS_DONE] = 1.0;
            sc[KS_STATUS] = 2.0;
        }
        return;
    }
    double alpha = sc[KS_RZ] / pq;
    double a0 = 0, a1 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        double ri = r[i] - alpha * q[i];
        r[i] = ri;
        double zi = ri / d[i];
        z[i] = zi;
        a0 += ri * zi;
        a1 += ri * ri;
    }
    part_store(part, KP_RHR, a0, sm);
    part_store(part, KP_RR, a1, sm);
}

// C3: beta = rz'/rz; p = z + beta p
__global__ void __launch_bounds__(KRY_T) k_cg_p(int n, const double* __restrict__ z, double* p, double* part,
                                                double* sc) {
    __shared__ double sm[32];
    if (sc[KS_DONE] != 0.0) return;
    double rz_new = part_total(part, KP_RHR, sm);
    double beta = rz_new / sc[KS_RZ];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = z[i] + beta * p[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) sc[KS_RZ_NEW] = rz_new;
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
// features and their squares; mode 1 sums (x - p_prev)^2 of the solution.
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
            double dp = K.x[i] - K.pprev[i];
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

// training pairs: target = (x - p_prev) / scale, weight = 1 / rows on solved rows
template <typename R>
__global__ void k_mlp_targets(int n, KryWork<R> K) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool on = K.kcnt[i] > 0;
    double rows = K.mstat[MS_ROWS];
    K.target[i] = on ? (float)((K.x[i] - K.pprev[i]) / K.mstat[MS_PS]) : 0.f;
    K.weight[i] = (on && rows > 0) ? (float)(1.0 / rows) : 0.f;
}

__global__ void k_mlp_tick(double* mstat) { mstat[MS_T] += 1.0; }

// ---- minimal-residual blend of the initial iterate ---------------------------
// x0 = p_prev + sum_k c_k d_k with the directions d0 = the network's
// predicted change (scale * y), d1 = the last pressure change, d2 = the
// one-sweep increment; c minimises ||r0 - sum_k c_k A d_k|| with
// r0 = b - A p_prev, so x0 is never worse (in residual) than p_prev.
constexpr int BLEND_N = 3;
template <typename R>
__global__ void k_blend_dirs(int n, KryWork<R> K, const R* __restrict__ dpres, double* d0, double* d1, double* d2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool on = K.kcnt[i] > 0;
    d0[i] = on ? K.mstat[MS_PS] * (double)K.yp[i] : 0.0;
    d1[i] = on ? (double)dpres[i] : 0.0;
    d2[i] = on ? (double)K.fraw[(size_t)i * MLP_FEAT + 2] : 0.0;
}
// r0 = b - A p_prev (A p_prev in y); block partials of (Ad_k, Ad_l), (Ad_k, r0)
__global__ void __launch_bounds__(KRY_T) k_blend_dots(int n, const double* __restrict__ b, const double* __restrict__ y,
                                                      const double* __restrict__ a0, const double* __restrict__ a1,
                                                      const double* __restrict__ a2, double* part) {
    __shared__ double sm[32];
    double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double r0 = b[i] - y[i], u0 = a0[i], u1 = a1[i], u2 = a2[i];
        g[0] += u0 * u0; g[1] += u0 * u1; g[2] += u0 * u2;
        g[3] += u1 * u1; g[4] += u1 * u2; g[5] += u2 * u2;
        g[6] += u0 * r0; g[7] += u1 * r0; g[8] += u2 * r0;
    }
    for (int q = 0; q < 9; q++) {
        double t = block_sum(g[q], sm);
        if (threadIdx.x == 0) part[q * KRY_G + blockIdx.x] = t;
    }
}
// one block: totals, then the 3x3 least-squares solve (Gaussian elimination
// with a relative Tikhonov floor on the diagonal); c = 0 for a degenerate set
__global__ void __launch_bounds__(KRY_T) k_blend_solve(const double* part, double* sc) {
    __shared__ double sm[32];
    __shared__ double g[9];
    for (int q = 0; q < 9; q++) {
        double t = part_total(part, q, sm);
        if (threadIdx.x == 0) g[q] = t;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double A[3][4] = {{g[0], g[1], g[2], g[6]}, {g[1], g[3], g[4], g[7]}, {g[2], g[4], g[5], g[8]}};
    double tr = g[0] + g[3] + g[5];
    double c[3] = {0, 0, 0};
    if (tr > 0 && isfinite(tr)) {
        for (int k = 0; k < 3; k++) A[k][k] += 1e-12 * tr;
        bool ok = true;
        for (int k = 0; k < 3 && ok; k++) {
            int piv = k;
            for (int r = k + 1; r < 3; r++)
                if (fabs(A[r][k]) > fabs(A[piv][k])) piv = r;
            if (!(fabs(A[piv][k]) > 0)) { ok = false; break; }
            for (int q = 0; q < 4; q++) { double t = A[k][q]; A[k][q] = A[piv][q]; A[piv][q] = t; }
            for (int r = k + 1; r < 3; r++) {
                double f = A[r][k] / A[k][k];
                for (int q = k; q < 4; q++) A[r][q] -= f * A[k][q];
            }
        }
        if (ok) {
            for (int k = 2; k >= 0; k--) {
                double t = A[k][3];
                for (int q = k + 1; q < 3; q++) t -= A[k][q] * c[q];
                c[k] = t / A[k][k];
            }
            if (!(isfinite(c[0]) && isfinite(c[1]) && isfinite(c[2]))) c[0] = c[1] = c[2] = 0;
        }
    }
    sc[KS_C0] = c[0];
    sc[KS_C1] = c[1];
    sc[KS_C2] = c[2];
}
template <typename R>
__global__ void k_blend_apply(int n, KryWork<R> K, const double* __restrict__ d0, const double* __restrict__ d1,
                              const double* __restrict__ d2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || K.kcnt[i] == 0) return;
    K.x[i] = K.pprev[i] + K.sc[KS_C0] * d0[i] + K.sc[KS_C1] * d1[i] + K.sc[KS_C2] * d2[i];
}

// p_new = x on solved rows, the current pressure elsewhere
template <typename R>
__global__ void __launch_bounds__(128) k_kry_final(DevParams P, SphState<R> S, SphWork<R> W, KryWork<R> K) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.ns) return;
    bool solve = kry_solve_row(P, S.itype[i], S.ptype[i], S.btype[i]);
    R pold = W.rec.up[i].w;
    W.p_new[i] = solve ? (R)K.x[i] : pold;
    S.dpres[i] = solve ? (R)(K.x[i] - (double)pold) : (R)0;
}

}  // namespace sphdem
