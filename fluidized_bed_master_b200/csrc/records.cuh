// records.cuh -- packed per-particle records read by the neighbour passes.
//
// A neighbour pass reads a handful of fields of every neighbour j.  Read
// from separate SoA arrays that is one scattered load (and one 32-byte
// sector) per field and neighbour; the passes were bound by the latency of
// those loads.  The records below put what a pass reads of j into one or
// two aligned vectors, so a neighbour costs 2-4 vector loads:
//
//   PosRec  position + type tag      written by the cell gather (NNPS)
//     FP32 build: int4 {qx, qy, qz, tag}; q = round((x - o) / s) with the
//       origin o at the centre of the cell-grid box and s = extent / 2^30
//       per axis.  Differences of two fixed-point positions are exact
//       integers; one int->float conversion and a multiply give the
//       displacement with an absolute error below s (3.7e-10 m on a 0.4 m
//       axis), against 6e-8 relative for rounding a double difference.
//       Positions farther than one extent from the centre set the OOR tag
//       bit; pairs with that bit take their displacement from the double
//       positions.
//     FP64 build: {double x, y, z; int tag}: the exact double positions.
//   tag = p_type << 16 | buffer_type << 5 | OOR << 4 | i_type
//   MR0  {m, rho}                      start of step (cell gather)
//   F1   {m_new, rho_new, temp, DEMpor} pass A; walls' rho_new is patched by
//                                      the Neumann wall pass
//   UP   {ux, uy, uz, pres}            cell gather; u* by the SPH predictor,
//                                      wall pressure by the first Neumann pass
//   UT   {ux, uy, uz, temp}            corrector (pass C), patched by the
//                                      open-boundary pass for buffer particles
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "device_common.cuh"

namespace sphdem {

struct __align__(32) Dbl4 {
    double x, y, z, w;
};
struct __align__(32) QPos64 {
    double x, y, z;
    int w, pad;
};

template <typename R>
struct Vec;
template <>
struct Vec<float> {
    typedef float4 v4;
    typedef float2 v2;
    typedef int4 pos;
};
template <>
struct Vec<double> {
    typedef Dbl4 v4;
    typedef double2 v2;
    typedef QPos64 pos;
};

template <typename R>
using V4 = typename Vec<R>::v4;
template <typename R>
using V2 = typename Vec<R>::v2;
template <typename R>
using PosRec = typename Vec<R>::pos;

// ---- tag -----------------------------------------------------------------
constexpr int TAG_OOR = 1 << 4;
__host__ __device__ __forceinline__ int make_tag(int ptype, int btype, int itype, int oor) {
    return (int)((unsigned)ptype << 16) | ((btype & 7) << 5) | (oor ? TAG_OOR : 0) | (itype & 15);
}
__device__ __forceinline__ int tag_ptype(int t) { return t >> 16; }
__device__ __forceinline__ int tag_btype(int t) { return (t >> 5) & 7; }
__device__ __forceinline__ int tag_itype(int t) { return t & 15; }

// ---- vector loads / stores (read-only path for the neighbour loads) ------
__device__ __forceinline__ float4 ldr(const float4* p) { return __ldg(p); }
__device__ __forceinline__ float2 ldr(const float2* p) { return __ldg(p); }
__device__ __forceinline__ int4 ldr(const int4* p) { return __ldg(p); }
__device__ __forceinline__ double2 ldr(const double2* p) { return __ldg(p); }
__device__ __forceinline__ Dbl4 ldr(const Dbl4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return Dbl4{a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ QPos64 ldr(const QPos64* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    QPos64 r;
    r.x = a.x; r.y = a.y; r.z = b.x;
    r.w = __double_as_longlong(b.y) & 0xffffffff;
    r.pad = 0;
    return r;
}
// plain (coherent) loads for records written earlier in the same kernel
__device__ __forceinline__ float4 ldc(const float4* p) { return *p; }
__device__ __forceinline__ Dbl4 ldc(const Dbl4* p) { return *p; }

template <typename R>
__device__ __forceinline__ V4<R> mk4(R a, R b, R c, R d);
template <>
__device__ __forceinline__ float4 mk4<float>(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
template <>
__device__ __forceinline__ Dbl4 mk4<double>(double a, double b, double c, double d) { return Dbl4{a, b, c, d}; }
template <typename R>
__device__ __forceinline__ V2<R> mk2(R a, R b);
template <>
__device__ __forceinline__ float2 mk2<float>(float a, float b) { return make_float2(a, b); }
template <>
__device__ __forceinline__ double2 mk2<double>(double a, double b) { return make_double2(a, b); }

// component pointers for single-field patches (walls, buffers)
template <typename R>
__device__ __forceinline__ R* comp(V4<R>* p, int i, int c) { return reinterpret_cast<R*>(p + i) + c; }

// ---- position records ------------------------------------------------------
__device__ __forceinline__ int quantize(double v, double o, double inv, int& oor) {
    double t = __dmul_rn(__dsub_rn(v, o), inv);
    if (!(fabs(t) < 1073741823.0)) {   // |t| < 2^30 - 1; NaN lands here too
        oor = 1;
        return 0;
    }
    return __double2int_rn(t);
}

template <typename R>
__device__ __forceinline__ PosRec<R> make_pos(const DevParams& P, double x, double y, double z, int ptype, int btype,
                                              int itype);
template <>
__device__ __forceinline__ int4 make_pos<float>(const DevParams& P, double x, double y, double z, int ptype, int btype,
                                                int itype) {
    int oor = 0;
    int qx = quantize(x, P.q_org[0], P.q_inv[0], oor);
    int qy = quantize(y, P.q_org[1], P.q_inv[1], oor);
    int qz = quantize(z, P.q_org[2], P.q_inv[2], oor);
    return make_int4(qx, qy, qz, make_tag(ptype, btype, itype, oor));
}
template <>
__device__ __forceinline__ QPos64 make_pos<double>(const DevParams& P, double x, double y, double z, int ptype,
                                                   int btype, int itype) {
    QPos64 q;
    q.x = x; q.y = y; q.z = z;
    q.w = make_tag(ptype, btype, itype, 0);
    q.pad = 0;
    return q;
}
__device__ __forceinline__ void store_pos(int4* p, int i, const int4& v) { p[i] = v; }
__device__ __forceinline__ void store_pos(QPos64* p, int i, const QPos64& v) {
    double2* q = reinterpret_cast<double2*>(p + i);
    q[0] = make_double2(v.x, v.y);
    q[1] = make_double2(v.z, __longlong_as_double((long long)(unsigned)v.w));
}

// displacement x_i - x_j in field precision
template <typename R>
struct Disp {
    R dx, dy, dz;
};
__device__ __forceinline__ Disp<float> disp(const DevParams& P, const int4& a, const int4& b, const double* X,
                                            const double* Y, const double* Z, int i, int j) {
    Disp<float> d;
    if (((a.w | b.w) & TAG_OOR) == 0) {
        d.dx = (float)(a.x - b.x) * P.q_step[0];
        d.dy = (float)(a.y - b.y) * P.q_step[1];
        d.dz = (float)(a.z - b.z) * P.q_step[2];
    } else {
        d.dx = (float)(X[i] - X[j]);
        d.dy = (float)(Y[i] - Y[j]);
        d.dz = (float)(Z[i] - Z[j]);
    }
    return d;
}
__device__ __forceinline__ Disp<double> disp(const DevParams&, const QPos64& a, const QPos64& b, const double*,
                                             const double*, const double*, int, int) {
    return Disp<double>{a.x - b.x, a.y - b.y, a.z - b.z};
}
// displacement from a point given in double (mirror points, DEM centres)
__device__ __forceinline__ Disp<float> disp_pt(const DevParams& P, const int4& qp, const int4& b, double px, double py,
                                               double pz, const double* X, const double* Y, const double* Z, int j) {
    if (((qp.w | b.w) & TAG_OOR) == 0)
        return Disp<float>{(float)(qp.x - b.x) * P.q_step[0], (float)(qp.y - b.y) * P.q_step[1],
                           (float)(qp.z - b.z) * P.q_step[2]};
    return Disp<float>{(float)(px - X[j]), (float)(py - Y[j]), (float)(pz - Z[j])};
}
__device__ __forceinline__ Disp<double> disp_pt(const DevParams&, const QPos64&, const QPos64& b, double px, double py,
                                                double pz, const double*, const double*, const double*, int) {
    return Disp<double>{px - b.x, py - b.y, pz - b.z};
}

// ---- exact pair predicate with a fixed-point prefilter -----------------
// in == (sqrt(dx^2+dy^2+dz^2) + add < Rr) evaluated in FP64 exactly as the
// reference writes it (no contraction).  The FP32 build first compares the
// squared fixed-point displacement with Rr^2 (1 -/+ band); its error is
// below 2.5e-6 relative plus 3.5 steps/Rr, and band = 2e-6 + 8 steps/Rr
// covers both, so only pairs inside the band take the FP64 evaluation.
// d and r2 come back in field precision for the caller's sums.
struct Band {
    float lo, hi;
};
__device__ __forceinline__ Band make_band(const DevParams& P, double Rr) {
    double b = 2e-6 + P.q_abs / Rr;
    double r2 = Rr * Rr;
    return Band{(float)(r2 * (1.0 - b)), (float)(r2 * (1.0 + b))};
}
__device__ __forceinline__ bool test_pair(const DevParams& P, const int4& a, const int4& b, double ax, double ay,
                                          double az, const double* X, const double* Y, const double* Z, int j,
                                          double Rr, double add, Band bd, Disp<float>& d, float& r2) {
    if (((a.w | b.w) & TAG_OOR) == 0) {
        d.dx = (float)(a.x - b.x) * P.q_step[0];
        d.dy = (float)(a.y - b.y) * P.q_step[1];
        d.dz = (float)(a.z - b.z) * P.q_step[2];
        r2 = d.dx * d.dx + d.dy * d.dy + d.dz * d.dz;
        if (r2 < bd.lo) return true;
        if (r2 > bd.hi) return false;
    } else {
        d.dx = (float)(ax - X[j]);
        d.dy = (float)(ay - Y[j]);
        d.dz = (float)(az - Z[j]);
        r2 = d.dx * d.dx + d.dy * d.dy + d.dz * d.dz;
    }
    return __dadd_rn(pair_dist(ax, ay, az, X[j], Y[j], Z[j]), add) < Rr;
}
// test_pair for the two forms of the predicate at once: in0 with add = 0,
// in20 with add = 1e-20 (in20 implies in0); one prefilter, one FP64 distance
__device__ __forceinline__ void test_pair2(const DevParams& P, const int4& a, const int4& b, double ax, double ay,
                                           double az, const double* X, const double* Y, const double* Z, int j,
                                           double Rr, Band bd, Disp<float>& d, float& r2, bool& in0, bool& in20) {
    if (((a.w | b.w) & TAG_OOR) == 0) {
        d.dx = (float)(a.x - b.x) * P.q_step[0];
        d.dy = (float)(a.y - b.y) * P.q_step[1];
        d.dz = (float)(a.z - b.z) * P.q_step[2];
        r2 = d.dx * d.dx + d.dy * d.dy + d.dz * d.dz;
        if (r2 < bd.lo) { in0 = in20 = true; return; }
        if (r2 > bd.hi) { in0 = in20 = false; return; }
    } else {
        d.dx = (float)(ax - X[j]);
        d.dy = (float)(ay - Y[j]);
        d.dz = (float)(az - Z[j]);
        r2 = d.dx * d.dx + d.dy * d.dy + d.dz * d.dz;
    }
    const double r = pair_dist(ax, ay, az, X[j], Y[j], Z[j]);
    in0 = __dadd_rn(r, 0.0) < Rr;
    in20 = __dadd_rn(r, 1e-20) < Rr;
}
__device__ __forceinline__ void test_pair2(const DevParams&, const QPos64&, const QPos64& b, double ax, double ay,
                                           double az, const double*, const double*, const double*, int, double Rr,
                                           Band, Disp<double>& d, double& r2, bool& in0, bool& in20) {
    d.dx = ax - b.x;
    d.dy = ay - b.y;
    d.dz = az - b.z;
    const double r = pair_dist(ax, ay, az, b.x, b.y, b.z);
    r2 = d.dx * d.dx + d.dy * d.dy + d.dz * d.dz;
    in0 = __dadd_rn(r, 0.0) < Rr;
    in20 = __dadd_rn(r, 1e-20) < Rr;
}
__device__ __forceinline__ bool test_pair(const DevParams&, const QPos64&, const QPos64& b, double ax, double ay,
                                          double az, const double*, const double*, const double*, int, double Rr,
                                          double add, Band, Disp<double>& d, double& r2) {
    d.dx = ax - b.x;
    d.dy = ay - b.y;
    d.dz = az - b.z;
    double r = pair_dist(ax, ay, az, b.x, b.y, b.z);
    r2 = d.dx * d.dx + d.dy * d.dy + d.dz * d.dz;
    return __dadd_rn(r, add) < Rr;
}

// ---- pair distance, reciprocal ----------------------------------------------
// r = |d| + 1e-20 and 1/r as the reference forms them
// (sqrt(dx^2+dy^2+dz^2) + 1e-20).  FP32: rsqrt (2 ulp) instead of an IEEE
// sqrt and divide; the self pair (d = 0) gives r = 1e-20, 1/r = 1e20.
__device__ __forceinline__ void rdist(float r2, float& r, float& rinv) {
    if (r2 > 0.f) {
        float s = rsqrtf(r2);
        r = r2 * s;
        rinv = s;
    } else {
        r = 1e-20f;
        rinv = 1e20f;
    }
}
__device__ __forceinline__ void rdist(double r2, double& r, double& rinv) {
    r = sqrt(r2) + 1e-20;
    rinv = 1.0 / r;
}
__device__ __forceinline__ float rcp(float a) { return __fdividef(1.0f, a); }
__device__ __forceinline__ double rcp(double a) { return 1.0 / a; }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }

// ---- smoothing kernel with per-particle constants -----------------------
// W and dW/dr of functions_KNL.cuh:2-144 with 1/h precomputed.
// KT is the kernel type when the kernel instantiation fixes it (3: Wendland
// C2, the loops then carry no type test), -1 when it is read from kt.
template <typename R, int KT = -1>
struct Knl {
    static_assert(KT == -1 || KT == 3, "kernel types fixed at compile time: Wendland C2");
    int kt;
    R tA, ih, th;   // normalisation, 1/h, h
};
template <typename R, int KT = -1>
__device__ __forceinline__ Knl<R, KT> knl_make(const DevParams& P, R th) {
    Knl<R, KT> k;
    k.kt = P.kernel_type;
    k.tA = knl_tmpA<R>(P.kernel_type, P.dim, th);
    k.ih = rcp(th);
    k.th = th;
    return k;
}
// The other kernel types (Gaussian, cubic/quintic splines, Wendland C4) are
// called out of line: inlined into every neighbour loop, their exp/pow
// code held registers and kept the loops from being scheduled well even
// when the Wendland branches run.
template <typename R>
__device__ __noinline__ R knl_w_call(int kt, R tA, R tH, R rr) {
    return knl_w<R>(kt, tA, tH, rr);
}
template <typename R>
__device__ __noinline__ R knl_dw_call(int kt, R tA, R tH, R rr) {
    return knl_dw<R>(kt, tA, tH, rr);
}
template <typename R, int KT>
__device__ __forceinline__ R kw(const Knl<R, KT>& k, R rr) {
    if (KT == 3 || k.kt == 3) {
        R q = rr * k.ih * (R)0.5;
        if (!(q < (R)1)) return (R)0;
        R a = (R)1 - q, a2 = a * a;
        return k.tA * a2 * a2 * ((R)1 + (R)4 * q);
    }
    if constexpr (KT == -1) {
        if (k.kt == 5) {
            R q = rr * k.ih * (R)0.5;
            if (!(q < (R)1)) return (R)0;
            R a = (R)1 - q, a2 = a * a, a4 = a2 * a2;
            return k.tA * a4 * a4 * ((R)1 + (R)8 * q + (R)25 * q * q + (R)32 * q * q * q);
        }
        return knl_w_call<R>(k.kt, k.tA, k.th, rr);
    }
    return (R)0;
}
template <typename R, int KT>
__device__ __forceinline__ R kdw(const Knl<R, KT>& k, R rr) {
    if (KT == 3 || k.kt == 3) {
        R q = rr * k.ih * (R)0.5;
        if (!(q < (R)1)) return (R)0;
        R a = (R)1 - q;
        return ((R)0.5 * k.ih) * k.tA * ((R)-20 * q * a * a * a);
    }
    if constexpr (KT == -1) {
        if (k.kt == 5) {
            R q = rr * k.ih * (R)0.5;
            if (!(q < (R)1)) return (R)0;
            R a = (R)1 - q, a2 = a * a, a4 = a2 * a2;
            return ((R)0.5 * k.ih) * k.tA * ((R)-22 * q * a4 * a2 * a * ((R)16 * q * q + (R)7 * q + (R)1));
        }
        return knl_dw_call<R>(k.kt, k.tA, k.th, rr);
    }
    return (R)0;
}

// ---- gradient correction with the matrix held in registers --------------
template <typename R>
struct Cm9 {
    R c[9];
};
template <typename R>
__device__ __forceinline__ Cm9<R> cm_load(const R* __restrict__ Cm, int n, int i, int on) {
    Cm9<R> m;
#pragma unroll
    for (int q = 0; q < 9; q++) m.c[q] = on ? Cm[(size_t)q * n + i] : (R)((q % 4) == 0);
    return m;
}
template <typename R>
__device__ __forceinline__ void cm_apply(const Cm9<R>& m, int on, R& ax, R& ay, R& az) {
    if (!on) return;
    R a = ax, b = ay, c = az;
    ax = m.c[0] * a + m.c[1] * b + m.c[2] * c;
    ay = m.c[3] * a + m.c[4] * b + m.c[5] * c;
    az = m.c[6] * a + m.c[7] * b + m.c[8] * c;
}

// neighbour record bundles loaded by the list passes
template <typename R>
struct NbQ2 {
    PosRec<R> q;
    V2<R> a;
};
template <typename R>
struct NbQ2S {
    PosRec<R> q;
    V2<R> a;
    R s;
};
template <typename R>
struct NbQ44 {
    PosRec<R> q;
    V4<R> a, b;
};
template <typename R>
struct NbQ24 {
    PosRec<R> q;
    V2<R> a;
    V4<R> b;
};

// ---- the SPH neighbour list ---------------------------------------------
// Blocks of 8 entries per particle: entry k of particle i at
// ((k / 8) n + i) 8 + k % 8.  A particle's 8 consecutive entries fill one
// 32-byte sector: the list build's stores of one particle land in the same
// sector (written back whole from L2) and a walk loads B entries in one
// vector load, while the particles of a warp (consecutive i) still read
// consecutive sectors.
__host__ __device__ __forceinline__ size_t nb_at(int k, int n, int i) {
    return ((size_t)(k >> 3) * n + i) * 8 + (k & 7);
}

// ---- batched neighbour-list walk -------------------------------------------
// The list passes are bound by the latency of the dependent loads (list
// entry -> neighbour records).  Loading the records of B neighbours before
// any of their arithmetic keeps B independent load chains in flight; the
// sums still run in list order.  B = 2 or 4 entries come in one vector load.
template <int B, typename T, typename L, typename C>
__device__ __forceinline__ void nb_walk(int cnt, const int* __restrict__ nb, int n, int i, L load, C comp) {
    static_assert(B == 2 || B == 4, "list walks load 2 or 4 entries at a time");
    int k = 0;
    for (; k + B <= cnt; k += B) {
        int j[B];
        T r[B];
        if constexpr (B == 4) {
            const int4 v = __ldg(reinterpret_cast<const int4*>(nb + nb_at(k, n, i)));
            j[0] = v.x; j[1] = v.y; j[2] = v.z; j[3] = v.w;
        } else {
            const int2 v = __ldg(reinterpret_cast<const int2*>(nb + nb_at(k, n, i)));
            j[0] = v.x; j[1] = v.y;
        }
#pragma unroll
        for (int u = 0; u < B; u++) r[u] = load(j[u]);
#pragma unroll
        for (int u = 0; u < B; u++) comp(j[u], r[u]);
    }
    for (; k < cnt; k++) {
        int j = __ldg(nb + nb_at(k, n, i));
        T r = load(j);
        comp(j, r);
    }
}

}  // namespace sphdem
