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
constexpr int KRY_NPART = 8;

// scalar slots
enum {
    KS_RHO = 0, KS_RHO_NEW, KS_ALPHA, KS_OMEGA, KS_BNORM, KS_RES, KS_DONE, KS_ITER, KS_RZ, KS_RZ_NEW,
    KS_TOL, KS_MAXIT, KS_STATUS, KS_COUNT = 16
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
};

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
// Same neighbour terms and source as k_ppe.  x0: the warm start (previous
// pressure, or the learned prediction when x0 != nullptr).
template <typename R>
__global__ void __launch_bounds__(128) k_kry_assemble(DevParams P, SphState<R> S, SphWork<R> W, KryWork<R> K,
                                                      const R* __restrict__ x0) {
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
            }
            K.a[(size_t)k * n + i] = acoef;
            k++;
        });
    R bsrc = (R)P.rho_gas * (bx + by + bz + (R)2 * S.dDEMpor[i] - W.dDEMpor_prev[i]) / (R)P.sdt;
    K.kcnt[i] = cnt;
    K.d[i] = dsum;
    K.b[i] = (double)bsrc + bfix;
    K.x[i] = x0 ? (double)x0[i] : (double)upi.w;
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

// p_new = x on solved rows, the current pressure elsewhere
template <typename R>
__global__ void __launch_bounds__(128) k_kry_final(DevParams P, SphState<R> S, SphWork<R> W, KryWork<R> K) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.ns) return;
    bool solve = kry_solve_row(P, S.itype[i], S.ptype[i], S.btype[i]);
    W.p_new[i] = solve ? (R)K.x[i] : W.rec.up[i].w;
}

}  // namespace sphdem
