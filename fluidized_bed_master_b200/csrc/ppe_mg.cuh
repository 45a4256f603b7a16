// ppe_mg.cuh -- two-level preconditioner for the PCG pressure solve
// (ppe_mode PCG with ppe_precond 1).  An engine extension: the reference
// has no converged PPE solver and no preconditioner.
//
// The PCG runs on A p = b with the m-weighted inner product <x, y> =
// sum m_i x_i y_i, in which A (a_ij = m_j g_ij with g symmetric) is
// self-adjoint: M A is symmetric positive definite.  The preconditioner is
//
//     z = D^-1 r  +  P0 V (P0^T M r)
//
// with D the diagonal of A (the Jacobi part the plain PCG already applies),
// P0 the piecewise-constant prolongation from the NNPS cells to their
// solved particles, and V a V-cycle for the cell operator
// A0 = P0^T (M A) P0.  Both terms are self-adjoint and positive in the
// m-weighted product, so the CG stays a CG.  The cell operator is a
// 27-point stencil on the cell grid (the neighbours of a particle lie in
// the 27 cells around its own); every coarser level aggregates 2x2x2 cells
// (Galerkin, again a 27-point stencil), down to at most MG_CHOL_MAX cells,
// which are solved exactly by their inverse, formed once per step from a
// Cholesky factor.  The
// V-cycle smooths with one damped-Jacobi sweep before and after the coarse
// correction (omega = MG_OMEGA), so it is a fixed symmetric operator.
//
// Per PCG iteration this adds the m-weighted restriction over the
// particles, the level-0 residual, one fused restriction-and-residual pass
// per coarser level, the last level's product with its inverse, one
// smoothing pass per level on the way up, the last of them fused with the
// prolongation into z; per step, the assembly of the cell operator from
// the stored coefficients, the Galerkin products and the inverse.
// No atomics: every sum has one owner and a fixed order, so a solve is
// bit-identical run to run.
#pragma once
#include "ppe_krylov.cuh"

namespace sphdem {

constexpr int MG_MAXLEV = 16;
constexpr int MG_CHOL_MAX = 64;
constexpr double MG_OMEGA = 0.7;

struct MgLevel {
    int nx, ny, nz, n;
    double* A;      // [n][32]: entry o = (dz+1)*9 + (dy+1)*3 + (dx+1) of cell c at A[c*32 + o]
    double* dinv;   // omega / A[13] (0 for a cell without solved particles)
    double *b;      // right-hand side
    double *x;      // the first damped-Jacobi sweep from zero, omega b / D
    double *t;      // down: residual b - A x; up: the level's correction
};

struct MgWork {
    int nlev;                  // levels 0..nlev-1; the last is solved by its inverse
    MgLevel L[MG_MAXLEV];
    double* chol;              // [MG_CHOL_MAX][MG_CHOL_MAX] inverse of the last level
    const int* key;            // cell of every particle slot (sorted keys)
    long long* cxyz;           // that cell's (x, y, z), 21 bits each (-1: no cell), formed per step
    const int* gs;             // first slot of every cell (-1: empty)
    const int* ge;
};

__device__ __forceinline__ void mg_xyz(const MgLevel& L, int c, int& x, int& y, int& z) {
    x = c % L.nx;
    y = (c / L.nx) % L.ny;
    z = c / (L.nx * L.ny);
}

// cell coordinates of every particle slot, so that the assembly finds a
// neighbour's stencil offset without divisions
__global__ void __launch_bounds__(256) k_mg_cellxyz(int n, MgWork M) {
    const MgLevel L0 = M.L[0];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = M.key[i];
    long long v = -1;
    if (c >= 0 && c < L0.n) {
        int x, y, z;
        mg_xyz(L0, c, x, y, z);
        v = (long long)x | ((long long)y << 21) | ((long long)z << 42);
    }
    M.cxyz[i] = v;
}

// A0 = P0^T (M A) P0 from the stored rows: one warp per cell, each lane
// adds its particles' rows into 27 partial sums, a fixed xor tree adds the
// lanes.  Row i of M A: m_i d_i on the diagonal, -m_i a_ij at each stored
// (solved) neighbour j.
template <typename R>
__global__ void __launch_bounds__(128) k_mg_assemble0(KryWork<R> K, MgWork M) {
    const MgLevel L0 = M.L[0];
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (c >= L0.n) return;
    double acc[27];
#pragma unroll
    for (int q = 0; q < 27; q++) acc[q] = 0.0;
    const int a0 = M.gs[c];
    if (a0 >= 0) {
        const int e0 = M.ge[c];
        int cx, cy, cz;
        mg_xyz(L0, c, cx, cy, cz);
        for (int i = a0 + lane; i < e0; i += 32) {
            const int cnt = K.kcnt[i];
            if (!cnt) continue;
            const double w = K.wm[i];
            acc[13] += w * K.d[i];
            for (int k = 0; k < cnt - 1; k++) {
                int j;
                double a;
                KEnt<R>::get(K.e[kent_at(i, k, K.cap)], j, a);
                const long long pj = M.cxyz[j];
                if (pj < 0) continue;
                const int dx = (int)(pj & 0x1FFFFF) - cx, dy = (int)((pj >> 21) & 0x1FFFFF) - cy,
                          dz = (int)(pj >> 42) - cz;
                if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) continue;
                acc[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] -= w * a;
            }
        }
    }
    double mine = 0.0;   // lane q keeps entry q
#pragma unroll
    for (int q = 0; q < 27; q++) {
        const double v = warp_sum(acc[q]);
        if (lane == q) mine = v;
    }
    if (lane < 27) L0.A[(size_t)c * 32 + lane] = mine;
    if (lane == 13) L0.dinv[c] = mine > 0.0 ? MG_OMEGA / mine : 0.0;
}

// Galerkin product for 2x2x2 aggregation: one thread per coarse cell adds
// its children's stencils; a child entry at offset o from child position
// (0/1 per axis) lands at the parent offset floor((child + o) / 2).
__global__ void __launch_bounds__(128) k_mg_coarsen(MgLevel F, MgLevel C) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= C.n) return;
    int X, Y, Z;
    mg_xyz(C, I, X, Y, Z);
    double s[27];
#pragma unroll
    for (int q = 0; q < 27; q++) s[q] = 0.0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const int cx = c & 1, cy = (c >> 1) & 1, cz = c >> 2;
        const int fx = 2 * X + cx, fy = 2 * Y + cy, fz = 2 * Z + cz;
        if (fx >= F.nx || fy >= F.ny || fz >= F.nz) continue;
        const int f = fx + F.nx * (fy + F.ny * fz);
#pragma unroll
        for (int o = 0; o < 27; o++) {
            const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = o / 9 - 1;
            const int px = (cx + ox) >> 1, py = (cy + oy) >> 1, pz = (cz + oz) >> 1;
            s[(pz + 1) * 9 + (py + 1) * 3 + (px + 1)] += F.A[(size_t)f * 32 + o];
        }
    }
#pragma unroll
    for (int q = 0; q < 27; q++) C.A[(size_t)I * 32 + q] = s[q];
    C.dinv[I] = s[13] > 0.0 ? MG_OMEGA / s[13] : 0.0;
}

// Inverse of the last level (n <= MG_CHOL_MAX), one CTA, once per step: the
// dense matrix of the stencil (rows of empty cells set to the identity),
// its Cholesky factor L, then A^-1 = L^-T L^-1 column by column, so that
// every application is one dense product.
__global__ void __launch_bounds__(256) k_mg_chol(MgLevel C, double* inv) {
    __shared__ double a[MG_CHOL_MAX][MG_CHOL_MAX + 1];
    const int n = C.n;
    for (int q = threadIdx.x; q < MG_CHOL_MAX * MG_CHOL_MAX; q += blockDim.x) a[q / MG_CHOL_MAX][q % MG_CHOL_MAX] = 0.0;
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        int x, yy, z;
        mg_xyz(C, r, x, yy, z);
        for (int o = 0; o < 27; o++) {
            const int jx = x + o % 3 - 1, jy = yy + (o / 3) % 3 - 1, jz = z + o / 9 - 1;
            if (jx < 0 || jy < 0 || jz < 0 || jx >= C.nx || jy >= C.ny || jz >= C.nz) continue;
            a[r][jx + C.nx * (jy + C.ny * jz)] = C.A[(size_t)r * 32 + o];
        }
        if (!(a[r][r] > 0.0)) a[r][r] = 1.0;
    }
    __syncthreads();
    for (int k = 0; k < n; k++) {
        if (threadIdx.x == 0) {
            double s = a[k][k];
            for (int j = 0; j < k; j++) s -= a[k][j] * a[k][j];
            a[k][k] = s > 0.0 ? sqrt(s) : 1.0;
        }
        __syncthreads();
        for (int r = k + 1 + threadIdx.x; r < n; r += blockDim.x) {
            double s = a[r][k];
            for (int j = 0; j < k; j++) s -= a[r][j] * a[k][j];
            a[r][k] = s / a[k][k];
        }
        __syncthreads();
    }
    // column c of the inverse: L y = e_c, L^T x = y, in place in inv; thread c owns column c
    const int c = threadIdx.x;
    if (c < n) {
        for (int k = 0; k < n; k++) {
            double s = k == c ? 1.0 : 0.0;
            for (int j = 0; j < k; j++) s -= a[k][j] * inv[j * MG_CHOL_MAX + c];
            inv[k * MG_CHOL_MAX + c] = s / a[k][k];
        }
        for (int k = n - 1; k >= 0; k--) {
            double s = inv[k * MG_CHOL_MAX + c];
            for (int j = k + 1; j < n; j++) s -= a[j][k] * inv[j * MG_CHOL_MAX + c];
            inv[k * MG_CHOL_MAX + c] = s / a[k][k];
        }
    }
}

// ---- one application: z += P0 V (P0^T M r) ------------------------------
// Down, level by level: b (restricted), x = omega b / D (the first sweep from
// zero), t = b - A x.  The last level: t = A^-1 b.  Up: t = x' + omega
// (b - A x') / D with x' = x + P t_coarser, formed where it is read, so no
// level is updated in place.

__device__ __forceinline__ int mg_nb(const MgLevel& C, int x, int y, int z, int o) {
    const int jx = x + o % 3 - 1, jy = y + (o / 3) % 3 - 1, jz = z + o / 9 - 1;
    if (jx < 0 || jy < 0 || jz < 0 || jx >= C.nx || jy >= C.ny || jz >= C.nz) return -1;
    return jx + C.nx * (jy + C.ny * jz);
}

// level 0: b[c] = sum over the cell's particles of m_i r_i, x = b omega / D
// (one warp per cell, lanes over its particles, a fixed xor tree)
__global__ void __launch_bounds__(128) k_mg_restrict0(const double* __restrict__ r, const double* __restrict__ wm,
                                                      MgWork M, const double* sc) {
    if (sc[KS_DONE] != 0.0) return;
    const MgLevel L0 = M.L[0];
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (c >= L0.n) return;
    double s = 0.0;
    const int a0 = M.gs[c];
    if (a0 >= 0) {
        const int e0 = M.ge[c];
        for (int i = a0 + lane; i < e0; i += 32) s += wm[i] * r[i];
    }
    s = warp_sum(s);
    if (lane == 0) {
        L0.b[c] = s;
        L0.x[c] = s * L0.dinv[c];
    }
}

// the stencil passes run one warp per cell (lane o takes neighbour o, a
// fixed xor tree adds them): the levels have too few cells for one thread
// each to hide the gathers' latency
__global__ void __launch_bounds__(128) k_mg_resid(MgLevel C, const double* sc) {
    if (sc[KS_DONE] != 0.0) return;
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, o = threadIdx.x & 31;
    if (I >= C.n) return;
    int x, y, z;
    mg_xyz(C, I, x, y, z);
    double v = 0.0;
    if (o < 27) {
        const int J = mg_nb(C, x, y, z, o);
        if (J >= 0) v = C.A[(size_t)I * 32 + o] * C.x[J];
    }
    v = warp_sum(v);
    if (o == 0) C.t[I] = C.b[I] - v;
}
__device__ __forceinline__ double mg_post_warp(const MgLevel& C, const MgLevel& Cc, int I, int o) {
    int x, y, z;
    mg_xyz(C, I, x, y, z);
    double v = 0.0, xp = 0.0;
    if (o < 27) {
        const int jx = x + o % 3 - 1, jy = y + (o / 3) % 3 - 1, jz = z + o / 9 - 1;
        if (jx >= 0 && jy >= 0 && jz >= 0 && jx < C.nx && jy < C.ny && jz < C.nz) {
            xp = C.x[jx + C.nx * (jy + C.ny * jz)] + Cc.t[(jx >> 1) + Cc.nx * ((jy >> 1) + Cc.ny * (jz >> 1))];
            v = C.A[(size_t)I * 32 + o] * xp;
        }
    }
    const double xc = __shfl_sync(0xffffffffu, xp, 13);
    v = warp_sum(v);
    return xc + (C.b[I] - v) * C.dinv[I];
}

// level 0 up, fused with the prolongation: t0[I] as k_mg_post, then
// z_i += t0[I] for the cell's solved particles
__global__ void __launch_bounds__(128) k_mg_post0(MgWork M, const int* __restrict__ kcnt, double* z,
                                                  const double* sc) {
    if (sc[KS_DONE] != 0.0) return;
    const MgLevel C = M.L[0], Cc = M.L[1];
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, o = threadIdx.x & 31;
    if (I >= C.n) return;
    const int a0 = M.gs[I];
    if (a0 < 0) return;
    const double t = mg_post_warp(C, Cc, I, o);
    const int e0 = M.ge[I];
    for (int i = a0 + o; i < e0; i += 32)
        if (kcnt[i]) z[i] += t;
}

__global__ void __launch_bounds__(128) k_mg_post(MgLevel C, MgLevel Cc, const double* sc) {
    if (sc[KS_DONE] != 0.0) return;
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, o = threadIdx.x & 31;
    if (I >= C.n) return;
    const double t = mg_post_warp(C, Cc, I, o);
    if (o == 0) C.t[I] = t;
}

// down one level, one warp per coarse cell I: lane o forms the right-hand
// side of neighbour J = I + o from J's children's residuals, its first
// sweep x_J = b_J omega / D_J and the product A_IJ x_J; lane 13 (J = I)
// keeps b_I and x_I; t_I = b_I - sum_J A_IJ x_J
__global__ void __launch_bounds__(128) k_mg_down(MgLevel F, MgLevel C, const double* sc) {
    if (sc[KS_DONE] != 0.0) return;
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, o = threadIdx.x & 31;
    if (I >= C.n) return;
    int x, y, z;
    mg_xyz(C, I, x, y, z);
    double v = 0.0, bj = 0.0, xj = 0.0;
    if (o < 27) {
        const int jx = x + o % 3 - 1, jy = y + (o / 3) % 3 - 1, jz = z + o / 9 - 1;
        if (jx >= 0 && jy >= 0 && jz >= 0 && jx < C.nx && jy < C.ny && jz < C.nz) {
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int fx = 2 * jx + (q & 1), fy = 2 * jy + ((q >> 1) & 1), fz = 2 * jz + (q >> 2);
                if (fx < F.nx && fy < F.ny && fz < F.nz) bj += F.t[fx + F.nx * (fy + F.ny * fz)];
            }
            xj = bj * C.dinv[jx + C.nx * (jy + C.ny * jz)];
            v = C.A[(size_t)I * 32 + o] * xj;
        }
    }
    const double bi = __shfl_sync(0xffffffffu, bj, 13);
    v = warp_sum(v);
    if (o == 13) {
        C.b[I] = bj;
        C.x[I] = xj;
    }
    if (o == 0) C.t[I] = bi - v;
}

// the last level (n <= MG_CHOL_MAX), one CTA: b from the children's
// residuals, t = A^-1 b
__global__ void __launch_bounds__(MG_CHOL_MAX) k_mg_last(MgLevel F, MgLevel C, const double* __restrict__ inv,
                                                         const double* sc) {
    if (sc[KS_DONE] != 0.0) return;
    __shared__ double b[MG_CHOL_MAX];
    const int I = threadIdx.x;
    if (I < C.n) {
        int X, Y, Z;
        mg_xyz(C, I, X, Y, Z);
        double s = 0.0;
        for (int q = 0; q < 8; q++) {
            const int fx = 2 * X + (q & 1), fy = 2 * Y + ((q >> 1) & 1), fz = 2 * Z + (q >> 2);
            if (fx < F.nx && fy < F.ny && fz < F.nz) s += F.t[fx + F.nx * (fy + F.ny * fz)];
        }
        b[I] = s;
    }
    __syncthreads();
    if (I < C.n) {
        double s = 0.0;
        for (int j = 0; j < C.n; j++) s += inv[I * MG_CHOL_MAX + j] * b[j];
        C.t[I] = s;
    }
}

}  // namespace sphdem
