// Slab exchange of a spatially sharded ISPH-DEM bed: device kernels that
// select the particles of a range of cell layers, pack their persistent
// state into records, park particles (i_type 3: outside every cell, skipped
// by every kernel, sorted behind all cells) and unpack received records
// into parked slots.
//
// The persistent state of a particle is what the next step's reorder reads
// (k_cells_gather_sph / k_cells_gather_dem): positions, h, velocities,
// mass, density, pressure, temperature, porosity rate, Shepard sum, types
// and id, and for a sphere also its angular velocity, temperatures, drag,
// heat rate and contact history.  Records carry every real value as a
// double (SPH temperature absolute), so a record moves between handles of
// either precision, and an FP32 value survives the round trip exactly.
#pragma once

#include "engine.cuh"

namespace sphdem {

// SPH record: 13 doubles | 4 ints | 2 ints padding = 128 bytes
constexpr int SLAB_SPH_D = 13, SLAB_SPH_I = 4, SLAB_SPH_BYTES = 128;
// DEM record: 22 doubles | 16x3 spring doubles | 5 ints | 16 partner ids |
// 1 int padding = 648 bytes
constexpr int SLAB_DEM_D = 22, SLAB_DEM_BYTES = 648;

// where the current (end-of-step) value of each persistent SPH field lives:
// the arrays the next reorder reads
template <typename R>
struct SphCur {
    double *x, *y, *z, *h;
    R *ux, *uy, *uz, *m, *rho, *pres, *temp, *dDEMpor, *flt_s;
    int *ptype, *btype, *itype, *pid;
    double t_ref;
};

// cell layer of a particle along axis (0 x, 1 y, 2 z), or -1 when parked
__device__ __forceinline__ int slab_layer(const DevParams& P, double x, double y, double z, int it, int axis) {
    if (it == 3) return -1;
    int ic, jc, kc;
    cell_ijk(P, x, y, z, ic, jc, kc);
    return axis == 0 ? ic : (axis == 1 ? jc : kc);
}

// flag[i] = 1 for the particles to select: mode 0 active with layer in
// [lo, hi); mode 1 parked
__global__ void k_slab_flag(DevParams P, int n, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const int* __restrict__ itype, int axis, int lo, int hi,
                            int mode, int* __restrict__ blk_cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool f = false;
    if (i < n) {
        int it = itype[i];
        if (mode == 1) f = it == 3;
        else {
            int l = slab_layer(P, x[i], y[i], z[i], it, axis);
            f = l >= lo && l < hi;
        }
    }
    int c = __syncthreads_count(f);
    if (threadIdx.x == 0) blk_cnt[blockIdx.x] = c;
}

// exclusive scan of the block counts (one block; nb <= 1024 * per)
__global__ void k_slab_scan(int nb, int* __restrict__ blk_cnt, int* __restrict__ total) {
    __shared__ int part[1024];
    int per = (nb + blockDim.x - 1) / blockDim.x;
    int b0 = threadIdx.x * per, s = 0;
    for (int b = b0; b < min(nb, b0 + per); b++) s += blk_cnt[b];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int t = 0; t < (int)blockDim.x; t++) {
            int v = part[t];
            part[t] = acc;
            acc += v;
        }
        *total = acc;
    }
    __syncthreads();
    int acc = part[threadIdx.x];
    for (int b = b0; b < min(nb, b0 + per); b++) {
        int v = blk_cnt[b];
        blk_cnt[b] = acc;
        acc += v;
    }
}

// write the selected slots in ascending order (at most cap of them)
__global__ void k_slab_compact(DevParams P, int n, const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, const int* __restrict__ itype, int axis, int lo,
                               int hi, int mode, const int* __restrict__ blk_off, int* __restrict__ slots, int cap) {
    __shared__ int wsum[32];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool f = false;
    if (i < n) {
        int it = itype[i];
        if (mode == 1) f = it == 3;
        else {
            int l = slab_layer(P, x[i], y[i], z[i], it, axis);
            f = l >= lo && l < hi;
        }
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[w] = __popc(m);
    __syncthreads();
    int base = blk_off[blockIdx.x];
    for (int k = 0; k < w; k++) base += wsum[k];
    if (f) {
        int pos = base + __popc(m & ((1u << lane) - 1u));
        if (pos < cap) slots[pos] = i;
    }
}

template <typename R>
__global__ void k_slab_export_sph(SphCur<R> C, const int* __restrict__ slots, int n, unsigned char* __restrict__ buf) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int i = slots[k];
    double* d = reinterpret_cast<double*>(buf + (size_t)k * SLAB_SPH_BYTES);
    d[0] = C.x[i]; d[1] = C.y[i]; d[2] = C.z[i]; d[3] = C.h[i];
    d[4] = (double)C.ux[i]; d[5] = (double)C.uy[i]; d[6] = (double)C.uz[i];
    d[7] = (double)C.m[i]; d[8] = (double)C.rho[i]; d[9] = (double)C.pres[i];
    d[10] = (double)C.temp[i] + C.t_ref;
    d[11] = (double)C.dDEMpor[i]; d[12] = (double)C.flt_s[i];
    int* q = reinterpret_cast<int*>(d + SLAB_SPH_D);
    q[0] = C.ptype[i]; q[1] = C.btype[i]; q[2] = C.itype[i]; q[3] = C.pid[i]; q[4] = 0; q[5] = 0;
}

template <typename R>
__global__ void k_slab_import_sph(SphCur<R> C, const int* __restrict__ slots, int n,
                                  const unsigned char* __restrict__ buf) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int i = slots[k];
    const double* d = reinterpret_cast<const double*>(buf + (size_t)k * SLAB_SPH_BYTES);
    C.x[i] = d[0]; C.y[i] = d[1]; C.z[i] = d[2]; C.h[i] = d[3];
    C.ux[i] = (R)d[4]; C.uy[i] = (R)d[5]; C.uz[i] = (R)d[6];
    C.m[i] = (R)d[7]; C.rho[i] = (R)d[8]; C.pres[i] = (R)d[9];
    C.temp[i] = (R)(d[10] - C.t_ref);
    C.dDEMpor[i] = (R)d[11]; C.flt_s[i] = (R)d[12];
    const int* q = reinterpret_cast<const int*>(d + SLAB_SPH_D);
    C.ptype[i] = q[0]; C.btype[i] = q[1]; C.itype[i] = q[2]; C.pid[i] = q[3];
}

// the DEM set is FP64 in every build: fields copy as they are
#define SLAB_DEM_FIELDS(X)                                                                                 \
    X(x) X(y) X(z) X(h) X(rad) X(ux) X(uy) X(uz) X(wx) X(wy) X(wz) X(m) X(rho) X(ri) X(temp) X(temp1)     \
    X(temp2) X(temp3) X(Fdx_df) X(Fdy_df) X(Fdz_df) X(Q_sd)

__global__ void k_slab_export_dem(DemState<double> D, int nd, const int* __restrict__ slots, int n,
                                  unsigned char* __restrict__ buf) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int i = slots[k];
    double* d = reinterpret_cast<double*>(buf + (size_t)k * SLAB_DEM_BYTES);
    int f = 0;
#define EXP(name) d[f++] = D.name[i];
    SLAB_DEM_FIELDS(EXP)
#undef EXP
    for (int s = 0; s < SPHDEM_NSLOT; s++)
        for (int c = 0; c < 3; c++) d[SLAB_DEM_D + 3 * s + c] = D.hds[((size_t)s * 3 + c) * nd + i];
    int* q = reinterpret_cast<int*>(d + SLAB_DEM_D + 3 * SPHDEM_NSLOT);
    q[0] = D.ptype[i]; q[1] = D.btype[i]; q[2] = D.itype[i]; q[3] = D.pid[i]; q[4] = D.dem_idx[i];
    for (int s = 0; s < SPHDEM_NSLOT; s++) q[5 + s] = D.hid[(size_t)s * nd + i];
    q[5 + SPHDEM_NSLOT] = 0;
}

__global__ void k_slab_import_dem(DemState<double> D, int nd, const int* __restrict__ slots, int n,
                                  const unsigned char* __restrict__ buf) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int i = slots[k];
    const double* d = reinterpret_cast<const double*>(buf + (size_t)k * SLAB_DEM_BYTES);
    int f = 0;
#define IMP(name) D.name[i] = d[f++];
    SLAB_DEM_FIELDS(IMP)
#undef IMP
    for (int s = 0; s < SPHDEM_NSLOT; s++)
        for (int c = 0; c < 3; c++) D.hds[((size_t)s * 3 + c) * nd + i] = d[SLAB_DEM_D + 3 * s + c];
    const int* q = reinterpret_cast<const int*>(d + SLAB_DEM_D + 3 * SPHDEM_NSLOT);
    D.ptype[i] = q[0]; D.btype[i] = q[1]; D.itype[i] = q[2]; D.pid[i] = q[3]; D.dem_idx[i] = q[4];
    for (int s = 0; s < SPHDEM_NSLOT; s++) D.hid[(size_t)s * nd + i] = q[5 + s];
}

// park the active particles whose layer along axis is outside [lo, hi)
__global__ void k_slab_keep(DevParams P, int n, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, int* __restrict__ itype, int axis, int lo, int hi) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int it = itype[i];
    if (it == 3) return;
    int l = slab_layer(P, x[i], y[i], z[i], it, axis);
    if (l < lo || l >= hi) itype[i] = 3;
}

}  // namespace sphdem
