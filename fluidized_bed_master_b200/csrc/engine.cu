// engine.cu -- host side of the B200 SPH-DEM step engine and its C ABI.
//
// The time loop of the reference (ISPH_Calc_seperate.cuh:905-975) calls
// SOPHIA_single_ISPH once per step; sphdem_step does the same work as one
// CUDA graph per step (captured once per step variant and replayed).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <set>
#include <string>
#include <type_traits>
#include <vector>

#include "handle.h"
#include "ppe_krylov.cuh"
#include "ppe_mg.cuh"
#include "mlp.h"
#include "wcsph2d.cuh"
#include "slab.cuh"

using namespace sphdem;

#define CK(call)                                     \
    do {                                             \
        cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) return SPHDEM_E_CUDA; \
    } while (0)

static const int TPB = 128;

// kernel slots for per-kernel timing
enum {
    KT_HASH_S, KT_SORT_S, KT_GATHER_S, KT_HASH_D, KT_SORT_D, KT_GATHER_D, KT_LIST, KT_PASSA, KT_DEMPREP, KT_PASSB,
    KT_DEMCONTACT, KT_DEMCOUPLING, KT_SPHCOUPLING, KT_NEUMANN0, KT_PPE, KT_NEUMANN, KT_PASSC, KT_DEMUPDATE,
    KT_OPENBC, KT_XSPH, KT_ROWS_S, KT_ROWS_D, KT_PPE_ASM, KT_PPE_WARM, KT_PPE_SOLVE, KT_PPE_TRAIN, KT_DLIST,
    // 2-D WCSPH step
    KT_W_PRED, KT_W_NNPS, KT_W_LIST, KT_W_KGC, KT_W_PREP, KT_W_CONT, KT_W_INTER, KT_W_CORR, KT_W_XSPH,
    KT_W_FINISH, KT_COUNT
};
static const char* KT_NAMES[KT_COUNT] = {
    "hash_sph", "sort_sph", "cells_gather_sph", "hash_dem", "sort_dem", "cells_gather_dem",
    "build_list", "passA", "dem_prep", "passB", "dem_contact", "dem_coupling", "sph_coupling", "neumann0",
    "ppe", "neumann", "passC", "dem_update", "open_bc", "xsph", "rows_sph", "rows_dem",
    "ppe.assemble", "ppe.warm_start", "ppe.iterations", "ppe.training", "build_dem_list",
    "w.predictor", "w.nnps", "w.list", "w.kgc", "w.prep", "w.continuity", "w.interaction", "w.corrector",
    "w.xsph", "w.finish"};

// Event records inside a captured step graph must be external event
// nodes (cudaEventRecordExternal); a plain record during capture only
// marks a dependency point.
static void record_event(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
    else cudaEventRecord(e, s);
}

// events around a kernel (group) on the stream it is launched on
struct KTimer {
    SphdemHandle* H;
    int k;
    cudaStream_t s;
    KTimer(SphdemHandle* h, int kk, cudaStream_t st = nullptr)
        : H(h), k(kk), s(st ? st : h->stream), on(h->timing && (h->time_only < 0 || h->time_only == kk)) {
        if (on) {
            record_event(H->ev_beg[k], s);
            H->ev_used[k] = 1;
        }
    }
    void stop() {
        if (on && !stopped) record_event(H->ev_end[k], s);
        stopped = true;
    }
    ~KTimer() { stop(); }
    bool on;
    bool stopped = false;
};
#define KTIME(k) KTimer kt_##__LINE__(H, k)
#define KTIME_ON(k, st) KTimer kt_##__LINE__(H, k, st)

// ---------------------------------------------------------------------------
// allocation
// ---------------------------------------------------------------------------
namespace {

struct Alloc {
    std::vector<void*> ptrs;
    bool ok = true;
    template <typename T>
    T* get(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
            ok = false;
            return nullptr;
        }
        cudaMemset(p, 0, sizeof(T) * (n ? n : 1));
        ptrs.push_back(p);
        return (T*)p;
    }
};

// scratch of the NNPS cell sort (cell_sort.cuh) for n keys on num_cells cells
CellSort alloc_cell_sort(Alloc& A, int num_cells, int n) {
    CellSort c;
    c.nb = num_cells + 1;
    c.ntiles = (c.nb + SORT_TILE - 1) / SORT_TILE;
    c.cnt = A.get<int>(c.nb);
    c.fill = A.get<int>(c.nb);
    c.start = A.get<int>(c.nb);
    c.tile_sum = A.get<int>(c.ntiles);
    c.tmp = A.get<int>(n);
    c.big_last = 0;
    c.blk = A.get<int>((n + 255) / 256 + 1);
    return c;
}

template <typename R>
struct EngineHost {
    Engine<R> E;
    KryWork<R> K{};          // PPE solver state (allocated for the Krylov modes)
    MlpNet net{};            // learned warm start (warm_start = WARM_MLP)
    bool has_mlp = false;
    int mlp_trained = 0;     // training steps taken
    Alloc A;
    int nb_cap = 0;
    // SPH list build: 1 = one thread per particle (k_build_list); 2, 4, 8 =
    // one warp per cell, that many cells per block (k_build_list_tiled, FP32)
    int list_mode = 1;
    // SPH -> DEM list: false = a warp per cell (k_build_dlist), true = a
    // thread per particle (k_build_dlist_pp); picked at commit by timing
    bool dlist_pp = false;
    size_t list_elems = 0;
    MgWork mg{};             // two-level PCG preconditioner (ppe_precond TWO_LEVEL)
    bool has_mg = false;
};

template <typename R>
void alloc_sph_state(Alloc& A, SphState<R>& S, int n) {
    S.x = A.get<double>(n); S.y = A.get<double>(n); S.z = A.get<double>(n); S.h = A.get<double>(n);
    S.ux = A.get<R>(n); S.uy = A.get<R>(n); S.uz = A.get<R>(n);
    S.m = A.get<R>(n); S.rho = A.get<R>(n); S.pres = A.get<R>(n); S.temp = A.get<R>(n);
    S.dDEMpor = A.get<R>(n); S.flt_s = A.get<R>(n); S.dpres = A.get<R>(n);
    S.ptype = A.get<int>(n); S.btype = A.get<int>(n); S.itype = A.get<int>(n); S.pid = A.get<int>(n);
}

template <typename R>
void alloc_dem_state(Alloc& A, DemState<double>& D, int n) {
    D.x = A.get<double>(n); D.y = A.get<double>(n); D.z = A.get<double>(n); D.h = A.get<double>(n);
    D.rad = A.get<double>(n);
    D.ux = A.get<R>(n); D.uy = A.get<R>(n); D.uz = A.get<R>(n);
    D.wx = A.get<R>(n); D.wy = A.get<R>(n); D.wz = A.get<R>(n);
    D.m = A.get<R>(n); D.rho = A.get<R>(n); D.ri = A.get<R>(n);
    D.temp = A.get<R>(n); D.temp1 = A.get<R>(n); D.temp2 = A.get<R>(n); D.temp3 = A.get<R>(n);
    D.Fdx_df = A.get<R>(n); D.Fdy_df = A.get<R>(n); D.Fdz_df = A.get<R>(n); D.Q_sd = A.get<R>(n);
    D.ptype = A.get<int>(n); D.btype = A.get<int>(n); D.itype = A.get<int>(n); D.pid = A.get<int>(n);
    D.dem_idx = A.get<int>(n);
    D.hid = A.get<int>((size_t)n * SPHDEM_NSLOT);
    D.hds = A.get<double>((size_t)n * SPHDEM_NSLOT * 3);
}

template <typename R>
void alloc_work(Alloc& A, SphWork<R>& W, DemWork<double>& DW, int ns, int nd, int ncells) {
    W.m_new = A.get<R>(ns); W.rho_new = A.get<R>(ns); W.rho_ref = A.get<R>(ns); W.DEMpor = A.get<R>(ns);
    W.dDEMpor_prev = A.get<R>(ns);
    W.Cm = A.get<R>((size_t)ns * 9);
    W.ftx = A.get<R>(ns); W.fty = A.get<R>(ns); W.ftz = A.get<R>(ns); W.ftot = A.get<R>(ns);
    W.fpx = A.get<R>(ns); W.fpy = A.get<R>(ns); W.fpz = A.get<R>(ns);
    W.pgfx = A.get<R>(ns); W.pgfy = A.get<R>(ns); W.pgfz = A.get<R>(ns);
    W.dtemp = A.get<R>(ns); W.temp0 = A.get<R>(ns); W.vist = A.get<R>(ns);
    W.ux0 = A.get<R>(ns); W.uy0 = A.get<R>(ns); W.uz0 = A.get<R>(ns);
    W.p_new = A.get<R>(ns);
    W.u_tmpx = A.get<R>(ns); W.u_tmpy = A.get<R>(ns); W.u_tmpz = A.get<R>(ns); W.temp_tmp = A.get<R>(ns);
    W.key_in = A.get<int>(ns); W.key_out = A.get<int>(ns); W.val_in = nullptr; W.val_out = A.get<int>(ns);
    W.g_str = A.get<int>(ncells + 1); W.g_end = A.get<int>(ncells + 1);
    W.rows = A.get<int4>(ncells);
    W.ncnt = A.get<int>(ns);
    W.ncntd = A.get<int>(ns);
    W.nbrd = nullptr;
    W.wall_idx = A.get<int>(ns); W.buf_idx = A.get<int>(ns); W.counters = A.get<int>(4);
    W.nbr = nullptr;
    W.rec.pos = A.get<PosRec<R>>(ns);
    W.rec.mr0 = A.get<V2<R>>(ns);
    W.rec.f1 = A.get<V4<R>>(ns);
    W.rec.up = A.get<V4<R>>(ns);
    W.rec.ut = A.get<V4<R>>(ns);
    DW.flt_s = A.get<double>(nd); DW.flt_sd = A.get<double>(nd); DW.flt_sd2 = A.get<double>(nd); DW.DEMpor = A.get<double>(nd);
    DW.ftx = A.get<double>(nd); DW.fty = A.get<double>(nd); DW.ftz = A.get<double>(nd);
    DW.tqx = A.get<double>(nd); DW.tqy = A.get<double>(nd); DW.tqz = A.get<double>(nd);
    DW.dtemp = A.get<double>(nd); DW.dtemp1 = A.get<double>(nd); DW.dtemp2 = A.get<double>(nd); DW.dtemp3 = A.get<double>(nd);
    DW.Fdx_b = A.get<double>(nd); DW.Fdy_b = A.get<double>(nd); DW.Fdz_b = A.get<double>(nd);
    DW.Fdx_da = A.get<double>(nd); DW.Fdy_da = A.get<double>(nd); DW.Fdz_da = A.get<double>(nd);
    DW.ux0 = A.get<double>(nd); DW.uy0 = A.get<double>(nd); DW.uz0 = A.get<double>(nd); DW.temp0 = A.get<double>(nd);
    DW.magf = A.get<double>(nd);
    DW.key_in = A.get<int>(nd); DW.key_out = A.get<int>(nd); DW.val_in = nullptr; DW.val_out = A.get<int>(nd);
    DW.g_str = A.get<int>(ncells + 1); DW.g_end = A.get<int>(ncells + 1);
    DW.rows = A.get<int4>(ncells);
    DW.nbs = A.get<int>((size_t)nd * DEM_SPH_CAP);
    DW.ncs = A.get<int>(nd);
    DW.dcs = A.get<double>((size_t)nd * 14);
    DW.dcf = A.get<int>(nd);
}


// ---------------------------------------------------------------------------
// host <-> device field transfer (conversion R <-> double on the host)
// ---------------------------------------------------------------------------
// (a field stored with an offset, see field_offset, holds value - off)
template <typename R>
int upload_real(R* dst, const double* src, int n, cudaStream_t s, double off = 0.0) {
    std::vector<R> tmp(n);
    for (int i = 0; i < n; i++) tmp[i] = (R)(src[i] - off);
    CK(cudaMemcpyAsync(dst, tmp.data(), sizeof(R) * n, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    return SPHDEM_OK;
}
template <typename R>
int download_real(double* dst, const R* src, int n, cudaStream_t s, double off = 0.0) {
    std::vector<R> tmp(n);
    CK(cudaMemcpyAsync(tmp.data(), src, sizeof(R) * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int i = 0; i < n; i++) dst[i] = (double)tmp[i] + off;
    return SPHDEM_OK;
}

// offset the ISPH-DEM engine stores a field with: the SPH temperature is
// kept as T - t_ref (DevParams::t_ref)
static double field_offset(const DevParams& P, int which, int field) {
    return (which == 0 && field == SPHDEM_F_TEMP) ? P.t_ref : 0.0;
}

// ---------------------------------------------------------------------------
// NNPS for one set; writes the sorted state into dst.
// ---------------------------------------------------------------------------
template <typename R>
int nnps_sph(SphdemHandle* H, EngineHost<R>* EH, int src, int dst, int64_t* nl) {
    Engine<R>& E = EH->E;
    DevParams& P = E.P;
    SphWork<R>& W = E.sw;
    cudaStream_t st = H->stream;
    int n = P.ns;
    if (n == 0) return SPHDEM_OK;
    SphState<R>& S = E.S[src];
    {
        KTIME(KT_HASH_S);
        CK((launch_pdl(k_hash, nblocks(n, TPB), TPB, 0, st, P, n, S.x, S.y, S.z, S.itype, W.key_in, E.cs_s.cnt)));
    }
    {
        KTIME(KT_SORT_S);
        CK(cell_sort(E.cs_s, n, W.key_in, W.val_out, W.key_out, W.g_str, W.g_end, st));
    }
    CK(cudaMemsetAsync(W.counters, 0, sizeof(int) * 4, st));
    SphGatherSrc<R> g;
    if (P.xsph) { g.ux = W.u_tmpx; g.uy = W.u_tmpy; g.uz = W.u_tmpz; g.temp = W.temp_tmp; }
    else { g.ux = S.ux; g.uy = S.uy; g.uz = S.uz; g.temp = S.temp; }
    g.m = W.m_new; g.rho = W.rho_new; g.pres = W.p_new;
    {
        KTIME(KT_GATHER_S);
        CK((launch_pdl(k_cells_gather_sph<R>, nblocks(n, TPB), TPB, 0, st, P, S, g, E.S[dst], W.rec, W.val_out, W.wall_idx,
                                                                W.buf_idx, W.counters, E.flags)));
    }
    {
        KTIME(KT_ROWS_S);
        CK((launch_pdl(k_rows, nblocks(P.NI * P.NJ * P.NK, TPB), TPB, 0, st, P, W.g_str, W.g_end, W.rows)));
    }
    *nl += 7;
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

template <typename R>
int nnps_dem(SphdemHandle* H, EngineHost<R>* EH, int src, int dst, int64_t* nl, cudaStream_t st) {
    Engine<R>& E = EH->E;
    DevParams& P = E.P;
    DemWork<double>& DW = E.dw;
    int n = P.nd;
    if (n == 0) {
        CK(cudaMemsetAsync(DW.g_str, 0xff, sizeof(int) * (P.num_cells + 1), st));
        CK(cudaMemsetAsync(DW.rows, 0, sizeof(int4) * P.NI * P.NJ * P.NK, st));
        return SPHDEM_OK;
    }
    DemState<double>& D = E.D[src];
    {
        KTIME_ON(KT_HASH_D, st);
        CK((launch_pdl(k_hash, nblocks(n, TPB), TPB, 0, st, P, n, D.x, D.y, D.z, D.itype, DW.key_in, E.cs_d.cnt)));
    }
    {
        KTIME_ON(KT_SORT_D, st);
        CK(cell_sort(E.cs_d, n, DW.key_in, DW.val_out, DW.key_out, DW.g_str, DW.g_end, st));
    }
    {
        KTIME_ON(KT_GATHER_D, st);
        CK((launch_pdl(k_cells_gather_dem<double>, nblocks(n, TPB), TPB, 0, st, P, D, E.D[dst], DW.val_out)));
        CK((launch_pdl(k_gather_history, nblocks(n * SPHDEM_NSLOT, TPB), TPB, 0, st, n, DW.val_out, D.hid, D.hds, E.D[dst].hid,
                                                                         E.D[dst].hds)));
    }
    {
        KTIME_ON(KT_ROWS_D, st);
        CK((launch_pdl(k_rows, nblocks(P.NI * P.NJ * P.NK, TPB), TPB, 0, st, P, DW.g_str, DW.g_end, DW.rows)));
    }
    *nl += 8;
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

// ---------------------------------------------------------------------------
// PPE to a relative residual (ppe_krylov.cuh).  Assembly and the initial
// residual are plain kernels; the iterations are the body of a conditional
// while node of the step graph (captured on a side stream into the node's
// body graph).  Without a graph the host drives the same body.
// ---------------------------------------------------------------------------
// two-level preconditioner: the cell operator and its coarse levels, once
// per step after the coefficients are assembled
template <typename R>
static void mg_setup(EngineHost<R>* EH, cudaStream_t st) {
    const MgWork& M = EH->mg;
    k_mg_cellxyz<<<nblocks(EH->E.P.ns, 256), 256, 0, st>>>(EH->E.P.ns, M);
    k_mg_assemble0<R><<<nblocks(M.L[0].n * 32, 128), 128, 0, st>>>(EH->K, M);
    for (int l = 1; l < M.nlev; l++) k_mg_coarsen<<<nblocks(M.L[l].n, 128), 128, 0, st>>>(M.L[l - 1], M.L[l]);
    k_mg_chol<<<1, 256, 0, st>>>(M.L[M.nlev - 1], M.chol);
}

// z += P0 V (P0^T M r): the coarse part of the preconditioner
template <typename R>
static void mg_apply(EngineHost<R>* EH, cudaStream_t st) {
    const MgWork& M = EH->mg;
    const KryWork<R>& K = EH->K;
    const int n0 = M.L[0].n;
    k_mg_restrict0<<<nblocks(n0 * 32, 128), 128, 0, st>>>(K.r, K.wm, M, K.sc);
    k_mg_resid<<<nblocks(n0 * 32, 128), 128, 0, st>>>(M.L[0], K.sc);
    const int nl = M.nlev;
    for (int l = 1; l < nl - 1; l++)
        k_mg_down<<<nblocks(M.L[l].n * 32, 128), 128, 0, st>>>(M.L[l - 1], M.L[l], K.sc);
    k_mg_last<<<1, MG_CHOL_MAX, 0, st>>>(M.L[nl - 2], M.L[nl - 1], M.chol, K.sc);
    for (int l = nl - 2; l >= 1; l--)
        k_mg_post<<<nblocks(M.L[l].n * 32, 128), 128, 0, st>>>(M.L[l], M.L[l + 1], K.sc);
    k_mg_post0<<<nblocks(n0 * 32, 128), 128, 0, st>>>(M, K.kcnt, K.z, K.sc);
}

template <typename R>
static void krylov_body(SphdemHandle* H, EngineHost<R>* EH, cudaStream_t st, cudaGraphConditionalHandle hnd,
                        int in_graph) {
    KryWork<R>& K = EH->K;
    const DevParams& P = EH->E.P;
    const int* nb = EH->E.sw.nbr;
    int n = P.ns;
    if (H->p.ppe_mode == SPHDEM_PPE_PCG) {
        // u in z, w in v, s in s
        k_cg_upd<<<KRY_G, KRY_T, 0, st>>>(n, K.d, K.z, K.v, K.p, K.s, K.x, K.r, K.sc);
        if (EH->has_mg) mg_apply<R>(EH, st);
        k_cg_spmv<R><<<KRY_GS, KRY_T, 0, st>>>(n, K, K.z, K.v, K.r, K.b, 0, hnd, in_graph);
    } else {
        k_bicg_p<<<KRY_G, KRY_T, 0, st>>>(n, K.d, K.r, K.p, K.v, K.y, K.part, K.sc);
        k_kry_spmv<R><<<KRY_G, KRY_T, 0, st>>>(n, K, nb, K.y, K.v, K.rh, KP_RHV, nullptr, 0, 0);
        k_bicg_s<<<KRY_G, KRY_T, 0, st>>>(n, K.d, K.r, K.v, K.y, K.x, K.s, K.z, K.part, K.sc);
        k_kry_spmv<R><<<KRY_G, KRY_T, 0, st>>>(n, K, nb, K.z, K.t, K.s, KP_TS, nullptr, KP_TT, 1);
        k_bicg_x<<<KRY_G, KRY_T, 0, st>>>(n, K.s, K.t, K.z, K.rh, K.x, K.r, K.part, K.sc);
        k_kry_check<<<1, KRY_T, 0, st>>>(K.part, K.sc, hnd, in_graph, 0);
    }
}

// learned warm start, before the solve: statistics (training steps),
// normalised features, and in use the network's predicted change (its
// direction in the projected initial iterate)
template <typename R>
static int mlp_before_solve(SphdemHandle* H, EngineHost<R>* EH, int phase) {
    KryWork<R>& K = EH->K;
    int n = EH->E.P.ns;
    cudaStream_t st = H->stream;
    if (phase == 1) {
        k_mlp_stats<R><<<KRY_G, KRY_T, 0, st>>>(n, K, 0);
        k_mlp_stats_final<R><<<1, KRY_T, 0, st>>>(KRY_G, K, 0);
    }
    k_mlp_norm<R><<<nblocks(n * MLP_FEAT, 256), 256, 0, st>>>(n, K);
    if (phase == 2) {
        int r = mlp_forward(EH->net, K.feat, n, K.yp, st);
        if (r) return r;
    }
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

// projected initial iterate (warm starts PROJECT and MLP): A p_prev, the
// directions, their products and dots in one pass, the small solve, x0
template <typename R>
static int project_initial(SphdemHandle* H, EngineHost<R>* EH, SphState<R>& S, int use_mlp, int cg) {
    KryWork<R>& K = EH->K;
    int n = EH->E.P.ns;
    cudaStream_t st = H->stream;
    const int nhist = std::min(std::max(H->p.warm_hist, 0), SPHDEM_WARM_HIST_MAX);
    k_proj_dirs<R><<<nblocks(n, 256), 256, 0, st>>>(n, K, S.pid, nhist, use_mlp);
    int fit = H->p.warm_fit | (cg ? 0 : SPHDEM_FIT_RESIDUAL);   // BiCGStab: the residual norm
    int pb = std::min(KRY_G, std::max(1, (n + PROJ_T - 1) / PROJ_T));
    switch (proj_groups(nhist)) {
    case 1: k_proj_spmv<R, 1><<<pb, PROJ_T, 0, st>>>(n, K, fit); break;
    case 2: k_proj_spmv<R, 2><<<pb, PROJ_T, 0, st>>>(n, K, fit); break;
    default: k_proj_spmv<R, 3><<<pb, PROJ_T, 0, st>>>(n, K, fit); break;
    }
    k_proj_solve<R><<<1, KRY_T, 0, st>>>(K, pb);
    k_proj_apply<R><<<nblocks(n, 256), 256, 0, st>>>(n, K, fit);
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

// learned warm start, after the solve (training steps): pressure scale,
// targets = scaled pressure change, mlp_updates Adam steps
template <typename R>
static int mlp_after_solve(SphdemHandle* H, EngineHost<R>* EH) {
    KryWork<R>& K = EH->K;
    int n = EH->E.P.ns;
    cudaStream_t st = H->stream;
    k_mlp_stats<R><<<KRY_G, KRY_T, 0, st>>>(n, K, 1);
    k_mlp_stats_final<R><<<1, KRY_T, 0, st>>>(KRY_G, K, 1);
    k_mlp_targets<R><<<nblocks(n, 256), 256, 0, st>>>(n, K);
    CK(cudaGetLastError());
    for (int u = 0; u < std::max(H->p.mlp_updates, 1); u++) {
        int r = mlp_grad(EH->net, K.feat, K.target, K.weight, n, 1.0f, st);
        if (r) return r;
        k_mlp_tick<<<1, 1, 0, st>>>(K.mstat);
        if ((r = mlp_adam(EH->net, (float)H->p.mlp_lr, 1, st, K.mstat + MS_T))) return r;
    }
    return SPHDEM_OK;
}

template <typename R>
static int enqueue_krylov(SphdemHandle* H, EngineHost<R>* EH, SphState<R>& S, SphWork<R>& W) {
    KryWork<R>& K = EH->K;
    const DevParams& P = EH->E.P;
    cudaStream_t st = H->stream;
    int n = P.ns;
    int cg = H->p.ppe_mode == SPHDEM_PPE_PCG;
    int phase = H->mlp_phase;
    CK(cudaMemsetAsync(K.sc + KS_DONE, 0, sizeof(double), st));
    {
        KTIME(KT_PPE_ASM);
        k_kry_assemble<R><<<nblocks(n, TPB), TPB, 0, st>>>(P, S, W, K, H->p.warm_start == SPHDEM_WARM_EXTRAPOLATE);
        if (EH->has_mg) mg_setup<R>(EH, st);
    }
    if (phase || K.D) {
        KTIME(KT_PPE_WARM);
        int r = phase ? mlp_before_solve<R>(H, EH, phase) : SPHDEM_OK;
        if (!r && K.D) r = project_initial<R>(H, EH, S, phase == 2, cg);
        if (r) return r;
    }
    KTimer kt_solve(H, KT_PPE_SOLVE);
    // y = A x0 (the projection already formed it from its kept products)
    if (!K.D) k_kry_spmv<R><<<KRY_G, KRY_T, 0, st>>>(n, K, W.nbr, K.x, K.y, K.x, KP_SS, nullptr, 0, 0);
    if (cg) {
        k_cg_init<<<KRY_G, KRY_T, 0, st>>>(n, K.d, K.b, K.y, K.r, K.z, K.p, K.s, K.sc, H->p.ppe_tol,
                                           H->p.ppe_max_iter);
        if (EH->has_mg) mg_apply<R>(EH, st);
        k_cg_spmv<R><<<KRY_GS, KRY_T, 0, st>>>(n, K, K.z, K.v, K.r, K.b, 1, 0, 0);
    } else {
        k_kry_init<<<KRY_G, KRY_T, 0, st>>>(n, K.d, K.b, K.y, K.r, K.rh, K.p, K.v, K.z, K.part, cg);
        k_kry_init_scalars<<<1, KRY_T, 0, st>>>(K.part, K.sc, H->p.ppe_tol, H->p.ppe_max_iter, cg);
    }
    CK(cudaGetLastError());
    if (H->capturing) {
        cudaStreamCaptureStatus cs;
        unsigned long long id = 0;
        cudaGraph_t cgraph = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(st, &cs, &id, &cgraph, &deps, &ndeps));
        if (cs != cudaStreamCaptureStatusActive) return SPHDEM_E_CUDA;
        cudaGraphConditionalHandle hnd;
        CK(cudaGraphConditionalHandleCreate(&hnd, cgraph, 1, cudaGraphCondAssignDefault));
        // (the union inside cudaGraphNodeParams has no default constructor)
        alignas(cudaGraphNodeParams) unsigned char cp_buf[sizeof(cudaGraphNodeParams)];
        std::memset(cp_buf, 0, sizeof(cp_buf));
        cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_buf);
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hnd;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, cgraph, deps, ndeps, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
        if (!H->side) CK(cudaStreamCreateWithFlags(&H->side, cudaStreamNonBlocking));
        CK(cudaStreamBeginCaptureToGraph(H->side, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        krylov_body<R>(H, EH, H->side, hnd, 1);
        cudaGraph_t out = nullptr;
        cudaError_t ce = cudaStreamEndCapture(H->side, &out);
        if (ce != cudaSuccess) return SPHDEM_E_CUDA;
    } else {
        double done = 0;
        for (int it = 0; it < std::max(H->p.ppe_max_iter, 1); it++) {
            krylov_body<R>(H, EH, st, 0, 0);
            CK(cudaMemcpyAsync(&done, K.sc + KS_DONE, sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (done != 0.0) break;
        }
    }
    kt_solve.stop();
    if (phase == 1) {
        KTIME(KT_PPE_TRAIN);
        int r = mlp_after_solve<R>(H, EH);
        if (r) return r;
    }
    k_kry_final<R><<<nblocks(n, TPB), TPB, 0, st>>>(P, S, W, K);
    if (K.hist) k_proj_ring<<<1, 1, 0, st>>>(K.hring);
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

// SPH -> DEM list of the sorted sets S, D (W.nbrd may be null: count only)
// The DEM contact, filter and coupling passes take a thread per sphere on
// 2-D beds with many spheres (a sphere there has a few DEM and ~70 SPH
// candidates, which a warp per sphere would leave mostly idle) and a warp
// per sphere otherwise (3-D beds, ~160 DEM candidates; and few spheres,
// where a warp each keeps more of the GPU busy).  A function of the
// configuration, so a given bed always runs one form.
inline bool dem_thread_per_sphere(const DevParams& P) { return P.dim == 2 && P.nd >= 65536; }

// warps of a grid-stride pass over the occupied cells of a sparse grid: at
// most one per SPH particle, at most 128 per SM
inline int occ_warps(const DevParams& P) { return std::max(1, std::min(P.ns, 148 * 128)); }

// the tiled wall pass (FP32): a warp per cell, or per occupied cell on a sparse grid
inline cudaError_t launch_neumann_tiled(Engine<float>& E, const SphState<float>& S, float* pres, int patch_up,
                                        cudaStream_t st) {
    const DevParams& P = E.P;
    SphWork<float>& W = E.sw;
    if (cell_sort_sparse(E.cs_s, P.ns))
        return launch_pdl(k_neumann_tiled<true>, (occ_warps(P) + NT_WARPS - 1) / NT_WARPS, NT_WARPS * 32, 0, st, P,
                          S, W, pres, (const int*)W.g_str, (const int*)W.g_end, (const int4*)W.rows, patch_up,
                          (const int*)E.cs_s.occ, (const int*)E.cs_s.occ_n);
    return launch_pdl(k_neumann_tiled<false>, (P.NI * P.NJ * P.NK + NT_WARPS - 1) / NT_WARPS, NT_WARPS * 32, 0, st,
                      P, S, W, pres, (const int*)W.g_str, (const int*)W.g_end, (const int4*)W.rows, patch_up,
                      (const int*)nullptr, (const int*)nullptr);
}

template <typename R>
cudaError_t launch_list(EngineHost<R>* EH, const SphState<R>& S, int mode, cudaStream_t st) {
    Engine<R>& E = EH->E;
    const DevParams& P = E.P;
    SphWork<R>& W = E.sw;
    if constexpr (std::is_same<R, float>::value) {
        if (mode == 2 || mode == 4 || mode == 8) {
            // slots outside every cell (i_type 3) keep an empty list
            cudaError_t e = cudaMemsetAsync(W.ncnt, 0, sizeof(int) * P.ns, st);
            if (e != cudaSuccess) return e;
            const int ncell = P.NI * P.NJ * P.NK;
            if (mode == 2)
                return launch_pdl(k_build_list_tiled<2>, (ncell + 1) / 2, 64, 0, st, P, S, W.rec, W.g_str, W.g_end,
                                  W.rows, W.nbr, W.ncnt, E.flags);
            if (mode == 4)
                return launch_pdl(k_build_list_tiled<4>, (ncell + 3) / 4, 128, 0, st, P, S, W.rec, W.g_str, W.g_end,
                                  W.rows, W.nbr, W.ncnt, E.flags);
            return launch_pdl(k_build_list_tiled<8>, (ncell + 7) / 8, 256, 0, st, P, S, W.rec, W.g_str, W.g_end,
                              W.rows, W.nbr, W.ncnt, E.flags);
        }
    }
    return launch_pdl(k_build_list<R>, nblocks(P.ns, TPB), TPB, 0, st, P, S, W.rec, W.rows, W.nbr, W.ncnt, E.flags);
}

// The list build of the step, picked per handle at commit (list_build 0):
// each candidate (one thread per particle; one warp per cell with 2, 4 or 8
// cells per block) builds the commit's list once untimed and three times
// timed, and the fastest is kept.  The candidates write the same lists, so
// the pick changes the speed only.  In two dimensions a cell holds a few
// particles and most lanes of a warp per cell idle; in the 3-D bed a cell
// holds ~23 and the warp shares the staged candidates.
template <typename R>
int tune_list_build(SphdemHandle* H, EngineHost<R>* EH, const SphState<R>& S) {
    if (!std::is_same<R, float>::value) {
        EH->list_mode = 1;
        return SPHDEM_OK;
    }
    if (H->list_build_req != 0) {
        EH->list_mode = H->list_build_req;
        return SPHDEM_OK;
    }
    cudaStream_t st = H->stream;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    const int cand[4] = {1, 2, 4, 8};
    float best = 0;
    int pick = 4;
    cudaError_t e = cudaSuccess;
    for (int c : cand) {
        if ((e = launch_list<R>(EH, S, c, st)) != cudaSuccess) break;
        if ((e = cudaEventRecord(a, st)) != cudaSuccess) break;
        for (int k = 0; k < 3 && e == cudaSuccess; k++) e = launch_list<R>(EH, S, c, st);
        if (e != cudaSuccess || (e = cudaEventRecord(b, st)) != cudaSuccess) break;
        if ((e = cudaEventSynchronize(b)) != cudaSuccess) break;
        float ms = 0;
        if ((e = cudaEventElapsedTime(&ms, a, b)) != cudaSuccess) break;
        if (c == cand[0] || ms < best) {
            best = ms;
            pick = c;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return SPHDEM_E_CUDA;
    EH->list_mode = pick;
    return SPHDEM_OK;
}

template <typename R>
cudaError_t launch_dlist(EngineHost<R>* EH, const SphState<R>& S, const DemState<double>& D, cudaStream_t st) {
    Engine<R>& E = EH->E;
    const DevParams& P = E.P;
    const int ncell = P.NI * P.NJ * P.NK;
    if (EH->dlist_pp)
        return launch_pdl(k_build_dlist_pp, nblocks(P.ns, TPB), TPB, 0, st, P, S.x, S.y, S.z, S.h,
                          (const int*)S.itype, (const int4*)E.dw.rows, D.x, D.y, D.z, (const int*)D.ptype, E.sw.nbrd,
                          E.sw.ncntd, P.nbd_cap, E.flags);
    if (cell_sort_sparse(E.cs_s, P.ns))   // the occupied cells, a warp each, grid-stride
        return launch_pdl(k_build_dlist<true>, (occ_warps(P) + DL_WARPS - 1) / DL_WARPS, DL_WARPS * 32, 0, st, P,
                          S.x, S.y, S.z, S.h, E.sw.g_str, E.sw.g_end, E.dw.rows, D.x, D.y, D.z, D.ptype, E.sw.nbrd,
                          E.sw.ncntd, P.nbd_cap, E.flags, (const int*)E.cs_s.occ, (const int*)E.cs_s.occ_n);
    return launch_pdl(k_build_dlist<false>, (ncell + DL_WARPS - 1) / DL_WARPS, DL_WARPS * 32, 0, st, P, S.x, S.y,
                      S.z, S.h, E.sw.g_str, E.sw.g_end, E.dw.rows, D.x, D.y, D.z, D.ptype, E.sw.nbrd, E.sw.ncntd,
                      P.nbd_cap, E.flags, (const int*)nullptr, (const int*)nullptr);
}

// The SPH -> DEM list build, picked at commit like the SPH list's: a thread
// per particle against a warp per cell (each once untimed, three times
// timed); both write the same list.  sphdem_set_list_build fixes it with
// the SPH list's mode (1: per particle; 2, 4, 8: per cell).
template <typename R>
int tune_dlist(SphdemHandle* H, EngineHost<R>* EH, const SphState<R>& S, const DemState<double>& D) {
    if (H->list_build_req != 0) {
        EH->dlist_pp = H->list_build_req == 1;
        return SPHDEM_OK;
    }
    cudaStream_t st = H->stream;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    float ms[2] = {0, 0};
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < 2 && e == cudaSuccess; c++) {
        EH->dlist_pp = c == 1;
        if ((e = launch_dlist<R>(EH, S, D, st)) != cudaSuccess) break;
        if ((e = cudaEventRecord(a, st)) != cudaSuccess) break;
        for (int k = 0; k < 3 && e == cudaSuccess; k++) e = launch_dlist<R>(EH, S, D, st);
        if (e != cudaSuccess || (e = cudaEventRecord(b, st)) != cudaSuccess) break;
        if ((e = cudaEventSynchronize(b)) != cudaSuccess) break;
        e = cudaEventElapsedTime(&ms[c], a, b);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return SPHDEM_E_CUDA;
    EH->dlist_pp = ms[1] < ms[0];
    return SPHDEM_OK;
}

// ---------------------------------------------------------------------------
// one step (SOPHIA_single_ISPH order).  flags: bit1 count==0, bit2 filter
// step, bit3 time==0.
//
// The DEM kernels that read no SPH pass run on a second stream, forked from
// and joined to the step stream by events (in the step graph: parallel
// branches):
//   step stream: SPH NNPS -> list -> [SPH->DEM list built] pass A -> pass B
//                -> [DEM prep done] DEM coupling -> SPH coupling -> walls, PPE,
//                pass C, open boundary, XSPH -> [DEM update done] tick
//   DEM stream:  DEM NNPS -> [SPH gathered] SPH->DEM list -> contact -> DEM prep
//                ... [SPH coupling done] DEM corrector + walls
// The SPH -> DEM list reads both sorted sets; the DEM contact reads only
// the DEM set; the DEM prep reads the gathered SPH records and the DEM set;
// the DEM corrector writes the DEM set after the SPH coupling has read it,
// and no later SPH kernel reads it.  Without
// both sets, or with sphdem_set_concurrency(h, 0), everything runs on the
// step stream in the same order.  The per-kernel timing events of a DEM
// kernel are recorded on its own stream.
// ---------------------------------------------------------------------------
enum { F_COUNT0 = 2, F_FILT = 4, F_TIME0 = 8 };

template <typename R>
int enqueue_step(SphdemHandle* H, EngineHost<R>* EH, int flags, int64_t* nl) {
    Engine<R>& E = EH->E;
    DevParams& P = E.P;
    SphWork<R>& W = E.sw;
    DemWork<double>& DW = E.dw;
    cudaStream_t st = H->stream;
    int ns = P.ns, nd = P.nd;
    int so = E.cur_s, sn = 1 - E.cur_s, dox = E.cur_d, dn = 1 - E.cur_d;
    int r;
    // Wendland C2 (the default): the neighbour passes are instantiated with
    // the kernel type fixed
    const bool kt3 = P.kernel_type == 3;
    // ... and, for the common switch set, with the switches fixed too
    const bool swc = kt3 && switch_set(P) == SW_COMMON;
    const bool fork = H->concurrent && ns > 0 && nd > 0 && H->dem_stream;
    cudaStream_t sd = fork ? H->dem_stream : st;
    // event k recorded on stream a / waited for on stream b (fork only)
    auto rec = [&](int k, cudaStream_t a) { return fork ? cudaEventRecord(H->fork_ev[k], a) : cudaSuccess; };
    auto wait = [&](int k, cudaStream_t b) { return fork ? cudaStreamWaitEvent(b, H->fork_ev[k], 0) : cudaSuccess; };
    CK(rec(0, st));
    CK(wait(0, sd));
    if ((r = nnps_dem<R>(H, EH, dox, dn, nl, sd))) return r;
    SphState<R>& S = E.S[sn];
    DemState<double>& D = E.D[dn];
    int bs = nblocks(ns, TPB), bd = nblocks(nd, TPB);
    int bdw = nblocks(nd * 32, TPB), bww = nblocks(P.nwall * 32, TPB), bbw = nblocks(P.nbuf * 32, TPB);
    if ((r = nnps_sph<R>(H, EH, so, sn, nl))) return r;
    CK(rec(2, st));   // SPH set gathered
    CK(wait(2, sd));
    if (ns > 0 && nd > 0) {
        KTIME_ON(KT_DLIST, sd);
        CK(launch_dlist<R>(EH, S, D, sd));
        *nl += 1;
    }
    CK(rec(1, sd));   // SPH -> DEM list built
    if (nd > 0) {
        {
            KTIME_ON(KT_DEMCONTACT, sd);
            if (dem_thread_per_sphere(P)) CK((launch_pdl(k_dem_contact<R, 1>, bd, TPB, 0, sd, P, D, DW, DW.rows, E.flags)));
            else CK((launch_pdl(k_dem_contact<R, 32>, bdw, TPB, 0, sd, P, D, DW, DW.rows, E.flags)));
        }
        {
            KTIME_ON(KT_DEMPREP, sd);   // see dem_thread_per_sphere
            if (dem_thread_per_sphere(P)) CK((launch_pdl(k_dem_prep<R, 1>, bd, TPB, 0, sd, P, S, W.rec, D, DW, W.rows, DW.rows)));
            else CK((launch_pdl(k_dem_prep<R, 32>, bdw, TPB, 0, sd, P, S, W.rec, D, DW, W.rows, DW.rows)));
        }
        *nl += 2;
    }
    if (ns > 0) {
        {
            KTIME(KT_LIST);
            CK(launch_list<R>(EH, S, EH->list_mode, st));
        }
        CK(wait(1, st));
        { KTIME(KT_PASSA); CK((launch_pdl(swc ? k_passA<R, 3, SW_COMMON> : kt3 ? k_passA<R, 3, -1> : k_passA<R, -1, -1>, bs, TPB, 0, st, P, S, W, D, DW.rows))); }
        *nl += 2;
        {
            KTIME(KT_PASSB);
            if (P.sps) {
                CK((launch_pdl(kt3 ? k_sps<R, 3> : k_sps<R, -1>, bs, TPB, 0, st, P, S, W)));
                *nl += 1;
            }
            if (P.iface | P.fb | P.sps | P.ipf) CK((launch_pdl(kt3 ? k_passB<R, true, 3, -1> : k_passB<R, true, -1, -1>, bs, TPB, 0, st, P, S, W, E.flags)));
            else CK((launch_pdl(swc ? k_passB<R, false, 3, SW_COMMON> : kt3 ? k_passB<R, false, 3, -1> : k_passB<R, false, -1, -1>, bs, TPB, 0, st, P, S, W, E.flags)));
        }
        *nl += 1;
    }
    CK(rec(3, sd));   // DEM contact and prep done
    CK(wait(1, st));  // (without SPH particles the list wait above was skipped)
    CK(wait(3, st));
    if (nd > 0) {
        {
            KTIME(KT_DEMCOUPLING);
            if (dem_thread_per_sphere(P))   // see dem_thread_per_sphere
                CK((launch_pdl(kt3 ? k_dem_coupling<R, 3, 1> : k_dem_coupling<R, -1, 1>, bd, TPB, 0, st, P, S, W, D, DW, W.rows)));
            else
                CK((launch_pdl(kt3 ? k_dem_coupling<R, 3, 32> : k_dem_coupling<R, -1, 32>, bdw, TPB, 0, st, P, S, W, D, DW, W.rows)));
            CK((launch_pdl(k_dem_finish<R>, bd, TPB, 0, st, P, D, DW)));
        }
        *nl += 2;
    }
    if (ns > 0) {
        KTIME(KT_SPHCOUPLING);
        CK((launch_pdl(kt3 ? k_sph_coupling<R, 3> : k_sph_coupling<R, -1>, bs, TPB, 0, st, P, S, W, D, DW, DW.rows, (flags & F_TIME0) ? 1 : 0)));
        *nl += 1;
    }
    CK(rec(4, st));   // the SPH coupling has read the DEM set
    CK(wait(4, sd));
    if (nd > 0) {
        { KTIME_ON(KT_DEMUPDATE, sd); CK((launch_pdl(k_dem_update<double>, bd, TPB, 0, sd, P, D, DW))); }
        *nl += 1;
    }
    if (ns > 0) {
        if (flags & F_COUNT0) {
            KTIME(KT_NEUMANN0);
            if constexpr (std::is_same<R, float>::value)
                CK(launch_neumann_tiled(E, S, S.pres, 1, st));
            else
                CK((launch_pdl(k_neumann<R>, bww, TPB, 0, st, P, S, W, S.pres, W.rows, 1)));
            *nl += 1;
        }
        {
            KTIME(KT_PPE);
            if (H->p.ppe_mode == SPHDEM_PPE_REFERENCE) CK((launch_pdl(swc ? k_ppe<R, 3, SW_COMMON> : kt3 ? k_ppe<R, 3, -1> : k_ppe<R, -1, -1>, bs, TPB, 0, st, P, S, W)));
            else if ((r = enqueue_krylov<R>(H, EH, S, W))) return r;
        }
        {
            KTIME(KT_NEUMANN);
            if constexpr (std::is_same<R, float>::value)
                CK(launch_neumann_tiled(E, S, W.p_new, 0, st));
            else
                CK((launch_pdl(k_neumann<R>, bww, TPB, 0, st, P, S, W, W.p_new, W.rows, 0)));
        }
        { KTIME(KT_PASSC); CK((launch_pdl(swc ? k_passC<R, 3, SW_COMMON> : kt3 ? k_passC<R, 3, -1> : k_passC<R, -1, -1>, bs, TPB, 0, st, P, S, W))); }
        *nl += 3;
        if (P.open_bc > 0) {
            KTIME(KT_OPENBC);
            CK((launch_pdl(kt3 ? k_open_bc<R, 3> : k_open_bc<R, -1>, bbw, TPB, 0, st, P, S, W, W.rows)));
            *nl += 1;
        }
        if (P.xsph) {
            KTIME(KT_XSPH);
            CK((launch_pdl(kt3 ? k_xsph<R, 3> : k_xsph<R, -1>, bs, TPB, 0, st, P, S, W)));
            *nl += 1;
        }
    }
    CK(rec(5, sd));   // join
    CK(wait(5, st));
    CK((launch_pdl(k_tick, 1, 1, 0, st, E.flags)));
    *nl += 1;
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

template <typename R>
int run_step(SphdemHandle* H, EngineHost<R>* EH, int64_t* nl) {
    Engine<R>& E = EH->E;
    int flags = 0;
    if (H->count == 0) flags |= F_COUNT0;
    if (H->time == 0.0) flags |= F_TIME0;
    H->mlp_phase = EH->has_mlp ? (EH->mlp_trained < H->p.mlp_train_steps ? 1 : 2) : 0;
    int key = flags | (E.cur_s << 8) | (E.cur_d << 9) | (H->mlp_phase << 10);
    int64_t n = 0;
    if (H->use_graphs) {
        auto it = H->graphs.find(key);
        if (it == H->graphs.end()) {
            cudaGraph_t g;
            if (H->timing) std::fill(H->ev_used.begin(), H->ev_used.end(), 0);
            CK(cudaStreamBeginCapture(H->stream, cudaStreamCaptureModeThreadLocal));
            H->capturing = true;
            int r = enqueue_step<R>(H, EH, flags, &n);
            H->capturing = false;
            cudaError_t ce = cudaStreamEndCapture(H->stream, &g);
            if (r) return r;
            if (ce != cudaSuccess) return SPHDEM_E_CUDA;
            cudaGraphExec_t ge;
            CK(cudaGraphInstantiate(&ge, g, 0));
            cudaGraphDestroy(g);
            H->graphs[key] = ge;
            H->graph_launches[key] = n;
            H->graph_kused[key] = H->ev_used;
            it = H->graphs.find(key);
        }
        n = H->graph_launches[key];
        if (H->timing) H->ev_used = H->graph_kused[key];
        CK(cudaGraphLaunch(it->second, H->stream));
    } else {
        int r = enqueue_step<R>(H, EH, flags, &n);
        if (r) return r;
    }
    *nl += n;
    E.cur_s ^= 1;
    E.cur_d ^= 1;
    if (H->mlp_phase == 1) EH->mlp_trained++;
    return SPHDEM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// commit: domain, grid, buffer tags, upload, list capacity
// ---------------------------------------------------------------------------
// bounding box: find_minmax (function_init.cuh:913-950) over the rows in
// file order, stopping one row short (the reference loop bound), then the
// margins; out = xmin, xmax, ymin, ymax, zmin, zmax
// the row of sphdem_set_beds (sorted by plane) whose plane is nearest y
static const SphdemBedRow& bed_row(const std::vector<SphdemBedRow>& rows, double y) {
    size_t k = std::upper_bound(rows.begin(), rows.end(), y,
                                [](double v, const SphdemBedRow& r) { return v < r.y; }) - rows.begin();
    if (k == 0) return rows[0];
    if (k == rows.size()) return rows[k - 1];
    return (std::fabs(rows[k].y - y) < std::fabs(rows[k - 1].y - y)) ? rows[k] : rows[k - 1];
}

static void bed_box(const SphdemParams& p, const double* fx, const double* fy, const double* fz, int n, double* out) {
    double mnx = fx[0], mxx = fx[0], mny = fy[0], mxy = fy[0], mnz = fz[0], mxz = fz[0];
    for (int k = 0; k < n - 1; k++) {
        mnx = std::min(mnx, fx[k]); mxx = std::max(mxx, fx[k]);
        mny = std::min(mny, fy[k]); mxy = std::max(mxy, fy[k]);
        mnz = std::min(mnz, fz[k]); mxz = std::max(mxz, fz[k]);
    }
    mnx -= (mxx - mnx) * p.margin[0]; mxx += (mxx - mnx) * p.margin[1];
    mny -= (mxy - mny) * p.margin[2]; mxy += (mxy - mny) * p.margin[3];
    mnz -= (mxz - mnz) * p.margin[4]; mxz += (mxz - mnz) * p.margin[5];
    out[0] = mnx; out[1] = mxx; out[2] = mny; out[3] = mxy; out[4] = mnz; out[5] = mxz;
}
template <typename R>
static int commit_t(SphdemHandle* H) {
    const SphdemParams& p = H->p;
    int ns = H->ns, nd = H->nd;
    // bounding box: find_minmax (function_init.cuh:913-950) over the rows in
    // file order, stopping one row short (the reference loop bound)
    std::vector<double> fx, fy, fz;
    double h0;
    if (H->have_file_order) {
        fx = H->file_x; fy = H->file_y; fz = H->file_z; h0 = H->file_h0;
    } else {
        auto& sx = H->stage_d[0][SPHDEM_F_X];
        auto& sy = H->stage_d[0][SPHDEM_F_Y];
        auto& sz = H->stage_d[0][SPHDEM_F_Z];
        auto& dx = H->stage_d[1][SPHDEM_F_X];
        auto& dy = H->stage_d[1][SPHDEM_F_Y];
        auto& dz = H->stage_d[1][SPHDEM_F_Z];
        fx = sx; fx.insert(fx.end(), dx.begin(), dx.end());
        fy = sy; fy.insert(fy.end(), dy.begin(), dy.end());
        fz = sz; fz.insert(fz.end(), dz.begin(), dz.end());
        h0 = ns > 0 ? H->stage_d[0][SPHDEM_F_H][0] : H->stage_d[1][SPHDEM_F_H][0];
    }
    double bb[6];
    bed_box(p, fx.data(), fy.data(), fz.data(), (int)fx.size(), bb);
    double mnx = bb[0], mxx = bb[1], mny = bb[2], mxy = bb[3], mnz = bb[4], mxz = bb[5];
    if (H->dom_set) {
        // a slab of a larger bed: the whole bed's box and h0, so that every
        // slab has the same cell grid
        mnx = H->dom_bbox[0]; mxx = H->dom_bbox[1]; mny = H->dom_bbox[2];
        mxy = H->dom_bbox[3]; mnz = H->dom_bbox[4]; mxz = H->dom_bbox[5];
        h0 = H->dom_h0;
    }
    double dcell = 1.1 * p.kappa * h0;
    int NI = (int)((mxx - mnx) / dcell) + 1, NJ = (int)((mxy - mny) / dcell) + 1, NK = (int)((mxz - mnz) / dcell) + 1;
    if (!(dcell > 0) || NI <= 0 || NJ <= 0 || NK <= 0 || (double)NI * NJ * NK > 2.0e9) return SPHDEM_E_INPUT;
    H->bbox[0] = mnx; H->bbox[1] = mxx; H->bbox[2] = mny; H->bbox[3] = mxy; H->bbox[4] = mnz; H->bbox[5] = mxz;
    H->nijk[0] = NI; H->nijk[1] = NJ; H->nijk[2] = NK;
    H->dcell = dcell;
    int num_cells = NI * NJ * NK + 1;
    // beds in planes y = const: no neighbour pair may cross two planes
    for (size_t b = 1; b < H->beds.size(); b++)
        if (!(H->beds[b].y - H->beds[b - 1].y > 2.0 * dcell)) return SPHDEM_E_INPUT;

    EngineHost<R>* EH = new EngineHost<R>();
    H->eng = EH;
    Engine<R>& E = EH->E;
    DevParams& P = E.P;
    std::memset(&P, 0, sizeof(P));
    P.kernel_type = p.kernel_type; P.dim = p.dim; P.kgc = p.kgc_solve; P.delsph = p.delSPH_solve;
    P.fp = p.fp_solve; P.fv = p.fv_solve; P.fva = p.fva_solve; P.fg = p.fg_solve; P.con = p.con_solve;
    P.iface = p.interface_solve; P.fb = p.fb_solve; P.c_repulsive = p.c_repulsive;
    P.sps = p.fv_solve == 1 && p.turbulence_model == 3;   // SPS (Parameters.cuh:111)
    P.ipf = p.fs_solve != 0 && p.surf_model == 1;         // Potential (inter-particle force)
    P.xsph = p.xsph_solve; P.open_bc = p.open_boundary; P.rho_type = p.rho_type;
    P.NI = NI; P.NJ = NJ; P.NK = NK; P.num_cells = num_cells;
    P.ns = ns; P.nd = nd;
    P.filt_period = p.freq_filt * p.decouple_stride;
    P.wall_mask = p.dem_wall_mask;
    P.sph_lagrangian = 0;   // KERNEL_set_alpha_sph: SPH particles are Eulerian (functions_ALE.cuh:26-47)
    P.kappa = p.kappa; P.dt = p.dt; P.sdt = p.decouple_stride * p.dt; P.soundspeed = p.soundspeed;
    P.u_limit = p.u_limit; P.c_xsph = p.c_xsph;
    P.xmin = mnx; P.xmax = mxx; P.ymin = mny; P.ymax = mxy; P.zmin = mnz; P.zmax = mxz;
    P.rho_gas = p.rho_gas; P.rho_liquid = p.rho_liquid; P.mu_gas = p.mu_gas; P.mu_liquid = p.mu_liquid;
    P.nu_gas = p.nu_gas; P.g_sph = p.g_sph; P.g_dem = p.g_dem; P.h_over_dx = p.h_over_dx;
    P.k_sph = p.k_sph; P.cp_sph = p.cp_sph; P.k_dem = p.k_dem; P.cp_dem = p.cp_dem;
    P.G = p.dem_shear_modulus; P.nu_p = p.dem_poisson; P.damp = p.dem_damp_coef; P.fric = p.dem_friction_ratio;
    P.r_contact = p.dem_contact_range; P.r_search = p.dem_search_range;
    P.inlet_uz = p.inlet_uz_mirror; P.inlet_temp = p.inlet_temp; P.L2 = p.obc_L2; P.L3 = p.obc_L3;
    P.ball_vel = p.ball_vel;
    if (!H->beds.empty()) {
        std::vector<double> rows;
        for (const SphdemBedRow& b : H->beds) {
            const double r[BED_COLS] = {b.y, b.inlet_uz, b.inlet_temp, b.obc_L2, b.obc_L3};
            rows.insert(rows.end(), r, r + BED_COLS);
        }
        CK(cudaMalloc(&H->d_beds, sizeof(double) * rows.size()));
        CK(cudaMemcpy(H->d_beds, rows.data(), sizeof(double) * rows.size(), cudaMemcpyHostToDevice));
        P.nbeds = (int)H->beds.size();
        P.beds = H->d_beds;
    }
    {
        // offset of the stored SPH temperature (DevParams::t_ref), an FP32 value
        auto& tv = H->stage_d[0][SPHDEM_F_TEMP];
        double s = 0;
        for (double v : tv) s += v;
        P.t_ref = tv.empty() ? 0.0 : (double)(float)(s / (double)tv.size());
        if (!std::isfinite(P.t_ref)) P.t_ref = 0.0;
        if (H->dom_set) P.t_ref = H->dom_tref;
    }
    P.cyl_cx = p.cyl_cx; P.cyl_cy = p.cyl_cy; P.cyl_r = p.cyl_r;
    for (int k = 0; k < 3; k++) { P.box_c[k] = p.box_c[k]; P.box_L[k] = p.box_L[k]; P.cone_c[k] = p.cone_c[k]; }
    P.cone_r1 = p.cone_r1; P.cone_r2 = p.cone_r2; P.cone_h = p.cone_h;
    P.rest_n = p.wall_rest_n; P.rest_s = p.wall_rest_s; P.mu_s = p.wall_mu_s; P.mu_rs = p.wall_mu_rs;
    // fixed-point position grid of the FP32 records: origin at the box
    // centre, 2^30 steps per box extent (records.cuh)
    {
        const double lo[3] = {mnx, mny, mnz}, hi[3] = {mxx, mxy, mxz};
        double smax = 0;
        for (int k = 0; k < 3; k++) {
            double e = hi[k] - lo[k];
            if (!(e > 0)) e = 1.0;
            double step = e / 1073741824.0;
            P.q_org[k] = 0.5 * (lo[k] + hi[k]);
            P.q_inv[k] = 1.0 / step;
            P.q_step[k] = (float)step;
            smax = std::max(smax, step);
        }
        P.q_abs = 8.0 * smax;
    }

    Alloc& A = EH->A;
    alloc_sph_state<R>(A, E.S[0], ns); alloc_sph_state<R>(A, E.S[1], ns);
    alloc_dem_state<double>(A, E.D[0], nd); alloc_dem_state<double>(A, E.D[1], nd);
    alloc_work<R>(A, E.sw, E.dw, ns, nd, num_cells);
    E.flags = A.get<DevFlags>(1);
    E.red_buf = A.get<double>(8);
    if (!A.ok) return SPHDEM_E_NOMEM;
    E.cur_s = 0; E.cur_d = 0;
    // cell sort scratch of both sets (zeroed by the allocator, as cell_sort expects)
    E.cs_s = alloc_cell_sort(A, num_cells, ns);
    // the occupied SPH cells, for the warp-per-cell passes on a sparse grid
    E.cs_s.occ = A.get<int>((size_t)ns + 1);
    E.cs_s.occ_n = A.get<int>(1);
    E.cs_d = alloc_cell_sort(A, num_cells, nd);
    // a slab's parked spare slots all sort into the last bucket
    E.cs_s.big_last = E.cs_d.big_last = H->dom_set ? 1 : 0;
    if (!A.ok) return SPHDEM_E_NOMEM;
    // buffer tags (c_initial_inner_outer_particle_single_{sph,dem}, functions_NNPS.cuh:60-200)
    // A slab of a larger bed (sphdem_set_domain) may pass i_type 3 for its
    // parked spare slots and its own ids (the rows' ids in the whole bed).
    for (int q = 0; q < 2; q++) {
        int nq = q ? nd : ns;
        std::vector<int> itype(nq, 1), btype(nq, 0), pid(nq);
        auto& pt = H->stage_i[q][SPHDEM_F_PTYPE];
        auto& zz = H->stage_d[q][SPHDEM_F_Z];
        const auto it_in = H->stage_i[q].find(SPHDEM_F_ITYPE);
        const auto pid_in = H->stage_i[q].find(SPHDEM_F_PID);
        const bool keep_it = H->dom_set && it_in != H->stage_i[q].end() && (int)it_in->second.size() == nq;
        const bool keep_pid = H->dom_set && pid_in != H->stage_i[q].end() && (int)pid_in->second.size() == nq;
        for (int i = 0; i < nq; i++) {
            pid[i] = keep_pid ? pid_in->second[i] : i;
            if (keep_it && it_in->second[i] == 3) {
                itype[i] = 3;
                continue;
            }
            if (p.open_boundary > 0 && pt[i] < 1000 && pt[i] >= 1) {
                double L1 = p.obc_L1, L2 = p.obc_L2, L3 = p.obc_L3, L4 = p.obc_L4;
                if (!H->beds.empty()) {
                    const SphdemBedRow& b = bed_row(H->beds, H->stage_d[q][SPHDEM_F_Y][i]);
                    L1 = b.obc_L1; L2 = b.obc_L2; L3 = b.obc_L3; L4 = b.obc_L4;
                }
                if (zz[i] >= (L1 - 1e-6) && (zz[i] < L2 - 1e-6)) { btype[i] = 1; itype[i] = 2; }
                if (zz[i] >= (L3 - 1e-6) && (zz[i] < L4 - 1e-6)) { btype[i] = 2; itype[i] = 2; }
            }
        }
        H->stage_i[q][SPHDEM_F_ITYPE] = itype;
        H->stage_i[q][SPHDEM_F_BUFFER_TYPE] = btype;
        H->stage_i[q][SPHDEM_F_PID] = pid;
    }
    {
        auto& pt = H->stage_i[0][SPHDEM_F_PTYPE];
        auto& bt = H->stage_i[0][SPHDEM_F_BUFFER_TYPE];
        auto& itv = H->stage_i[0][SPHDEM_F_ITYPE];
        int nw = 0, nb = 0;
        // the position records carry p_type in 16 bits
        for (int i = 0; i < ns; i++)
            if (pt[i] < -32768 || pt[i] > 32767) return SPHDEM_E_UNSUPPORTED;
        for (int i = 0; i < ns; i++) {
            if (itv[i] == 3) continue;
            if (pt[i] <= 0) nw++;
            if (bt[i] > 0 && pt[i] < 1000) nb++;
        }
        // launch bounds of the per-wall and per-buffer passes; the passes stop
        // at the step's own count.  A slab's membership changes every step:
        // headroom, and an overflow flag beyond it.
        if (H->dom_set) {
            nw = std::min(ns, nw + std::max(nw, 1024));
            nb = std::min(ns, nb + std::max(nb, 1024));
        }
        P.nwall = nw;
        P.nbuf = nb;
    }
    // DEM ids must be unique and >= 1: the contact history stores partner
    // ids and treats id < 1 as a free slot (functions_DEM_INTERACTION2.cuh:1326)
    if (nd > 0) {
        auto& id = H->stage_i[1][SPHDEM_F_DEM_IDX];
        std::set<int> seen;
        for (int v : id) {
            if (v < 1 || !seen.insert(v).second) return SPHDEM_E_INPUT;
        }
    }
    cudaStream_t st = H->stream;
    auto up_d = [&](double* dst, int q, int f, int nq) -> int {
        auto& v = H->stage_d[q][f];
        if ((int)v.size() != nq) v.assign(nq, 0.0);
        if (nq) CK(cudaMemcpyAsync(dst, v.data(), sizeof(double) * nq, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        return SPHDEM_OK;
    };
    auto up_r = [&](R* dst, int q, int f, int nq) -> int {
        auto& v = H->stage_d[q][f];
        if ((int)v.size() != nq) v.assign(nq, 0.0);
        return nq ? upload_real<R>(dst, v.data(), nq, st, field_offset(P, q, f)) : SPHDEM_OK;
    };
    auto up_i = [&](int* dst, int q, int f, int nq) -> int {
        auto& v = H->stage_i[q][f];
        if ((int)v.size() != nq) v.assign(nq, 0);
        if (nq) CK(cudaMemcpyAsync(dst, v.data(), sizeof(int) * nq, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        return SPHDEM_OK;
    };
    int r = 0;
    SphState<R>& S = E.S[0];
    SphWork<R>& W = E.sw;
    r |= up_d(S.x, 0, SPHDEM_F_X, ns); r |= up_d(S.y, 0, SPHDEM_F_Y, ns); r |= up_d(S.z, 0, SPHDEM_F_Z, ns);
    r |= up_d(S.h, 0, SPHDEM_F_H, ns);
    r |= up_r(S.ux, 0, SPHDEM_F_UX, ns); r |= up_r(S.uy, 0, SPHDEM_F_UY, ns); r |= up_r(S.uz, 0, SPHDEM_F_UZ, ns);
    r |= up_r(S.m, 0, SPHDEM_F_M, ns); r |= up_r(S.rho, 0, SPHDEM_F_RHO, ns); r |= up_r(S.pres, 0, SPHDEM_F_PRES, ns);
    r |= up_r(S.temp, 0, SPHDEM_F_TEMP, ns); r |= up_r(S.flt_s, 0, SPHDEM_F_FLT_S, ns);
    r |= up_r(S.dDEMpor, 0, SPHDEM_F_DDEMPOR, ns);
    r |= up_i(S.ptype, 0, SPHDEM_F_PTYPE, ns); r |= up_i(S.btype, 0, SPHDEM_F_BUFFER_TYPE, ns);
    r |= up_i(S.itype, 0, SPHDEM_F_ITYPE, ns); r |= up_i(S.pid, 0, SPHDEM_F_PID, ns);
    // end-of-step copies the reorder reads from
    r |= up_r(W.m_new, 0, SPHDEM_F_M, ns); r |= up_r(W.rho_new, 0, SPHDEM_F_RHO, ns);
    r |= up_r(W.p_new, 0, SPHDEM_F_PRES, ns);
    r |= up_r(W.u_tmpx, 0, SPHDEM_F_UX, ns); r |= up_r(W.u_tmpy, 0, SPHDEM_F_UY, ns);
    r |= up_r(W.u_tmpz, 0, SPHDEM_F_UZ, ns); r |= up_r(W.temp_tmp, 0, SPHDEM_F_TEMP, ns);
    DemState<double>& D = E.D[0];
    r |= up_d(D.x, 1, SPHDEM_F_X, nd); r |= up_d(D.y, 1, SPHDEM_F_Y, nd); r |= up_d(D.z, 1, SPHDEM_F_Z, nd);
    r |= up_d(D.h, 1, SPHDEM_F_H, nd); r |= up_d(D.rad, 1, SPHDEM_F_RAD, nd);
    r |= up_d(D.ux, 1, SPHDEM_F_UX, nd); r |= up_d(D.uy, 1, SPHDEM_F_UY, nd); r |= up_d(D.uz, 1, SPHDEM_F_UZ, nd);
    r |= up_d(D.wx, 1, SPHDEM_F_WX, nd); r |= up_d(D.wy, 1, SPHDEM_F_WY, nd); r |= up_d(D.wz, 1, SPHDEM_F_WZ, nd);
    r |= up_d(D.m, 1, SPHDEM_F_M, nd); r |= up_d(D.rho, 1, SPHDEM_F_RHO, nd); r |= up_d(D.ri, 1, SPHDEM_F_RI, nd);
    r |= up_d(D.temp, 1, SPHDEM_F_TEMP, nd); r |= up_d(D.temp1, 1, SPHDEM_F_TEMP1, nd);
    r |= up_d(D.temp2, 1, SPHDEM_F_TEMP2, nd); r |= up_d(D.temp3, 1, SPHDEM_F_TEMP3, nd);
    r |= up_d(D.Fdx_df, 1, SPHDEM_F_FDX_DF, nd); r |= up_d(D.Fdy_df, 1, SPHDEM_F_FDY_DF, nd);
    r |= up_d(D.Fdz_df, 1, SPHDEM_F_FDZ_DF, nd); r |= up_d(D.Q_sd, 1, SPHDEM_F_Q_SD, nd);
    r |= up_i(D.ptype, 1, SPHDEM_F_PTYPE, nd); r |= up_i(D.btype, 1, SPHDEM_F_BUFFER_TYPE, nd);
    r |= up_i(D.itype, 1, SPHDEM_F_ITYPE, nd); r |= up_i(D.pid, 1, SPHDEM_F_PID, nd);
    r |= up_i(D.dem_idx, 1, SPHDEM_F_DEM_IDX, nd);
    if (r) return SPHDEM_E_CUDA;
    // neighbour-list capacity from an exact count on the sorted input
    if (ns > 0) {
        int64_t nl = 0;
        P.nb_cap = 0;
        if ((r = nnps_sph<R>(H, EH, 0, 1, &nl))) return r;
        k_build_list<R><<<nblocks(ns, TPB), TPB, 0, st>>>(P, E.S[1], W.rec, W.rows, nullptr, W.ncnt, E.flags);
        CK(cudaGetLastError());
        DevFlags f;
        CK(cudaMemcpyAsync(&f, E.flags, sizeof(f), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        int cap = std::max(32, ((int)(f.max_ncnt * 1.25) + 16 + 7) / 8 * 8);
        P.nb_cap = cap;
        EH->nb_cap = cap;
        W.nbr = A.get<int>((size_t)cap * ns);
        if (!A.ok) return SPHDEM_E_NOMEM;
        if ((r = tune_list_build<R>(H, EH, E.S[1]))) return r;
        // SPH -> DEM list capacity from an exact count on the sorted input; a
        // particle above it later walks its stencil instead
        P.nbd_cap = 0;
        if (nd > 0) {
            if ((r = nnps_dem<R>(H, EH, 0, 1, &nl, st))) return r;
            CK(cudaMemsetAsync(W.ncntd, 0, sizeof(int) * ns, st));
            CK(launch_dlist<R>(EH, E.S[1], E.D[1], st));
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(&f, E.flags, sizeof(f), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            int capd = p.dem_list_cap > 0 ? p.dem_list_cap : std::max(8, ((int)(f.max_ncntd * 1.25) + 8 + 7) / 8 * 8);
            P.nbd_cap = capd;
            W.nbrd = A.get<int>((size_t)capd * ns);
            if (!A.ok) return SPHDEM_E_NOMEM;
            if ((r = tune_dlist<R>(H, EH, E.S[1], E.D[1]))) return r;
        }
        if (p.ppe_mode != SPHDEM_PPE_REFERENCE) {
            KryWork<R>& K = EH->K;
            K.e = A.get<typename KEnt<R>::T>((size_t)cap * ((ns + 31) / 32 * 32));
            K.cap = cap;
            K.ctr = A.get<unsigned>(1);
            K.wm = A.get<double>(ns);
            K.kcnt = A.get<int>(ns);
            double** vecs[] = {&K.d, &K.b, &K.x, &K.r, &K.rh, &K.p, &K.v, &K.s, &K.t, &K.y, &K.z};
            for (double** v : vecs) *v = A.get<double>(ns);
            K.part = A.get<double>((size_t)KRY_NPART * KRY_G);
            K.sc = A.get<double>(KS_COUNT);
            if (!A.ok) return SPHDEM_E_NOMEM;
            if (p.ppe_precond == SPHDEM_PRECOND_TWO_LEVEL) {
                // cell grid, then 2x2x2 aggregates down to at most MG_CHOL_MAX cells (two levels at least)
                MgWork& M = EH->mg;
                int nx = P.NI, ny = P.NJ, nz = P.NK, l = 0;
                while (true) {
                    MgLevel& L = M.L[l];
                    L.nx = nx; L.ny = ny; L.nz = nz; L.n = nx * ny * nz;
                    L.A = A.get<double>((size_t)32 * L.n);
                    L.dinv = A.get<double>(L.n);
                    L.b = A.get<double>(L.n); L.x = A.get<double>(L.n); L.t = A.get<double>(L.n);
                    l++;
                    if ((L.n <= MG_CHOL_MAX && l >= 2) || l == MG_MAXLEV) break;
                    nx = (nx + 1) / 2; ny = (ny + 1) / 2; nz = (nz + 1) / 2;
                }
                if (M.L[l - 1].n > MG_CHOL_MAX) return SPHDEM_E_UNSUPPORTED;
                M.nlev = l;
                M.chol = A.get<double>((size_t)MG_CHOL_MAX * MG_CHOL_MAX);
                M.key = W.key_out;
                M.cxyz = A.get<long long>(ns);
                M.gs = W.g_str;
                M.ge = W.g_end;
                if (!A.ok) return SPHDEM_E_NOMEM;
                EH->has_mg = true;
            }
            if (p.warm_start == SPHDEM_WARM_MLP || p.warm_start == SPHDEM_WARM_PROJECT) {
                K.D = A.get<float>((size_t)ns * PROJ_MP);
                K.hist = A.get<float>((size_t)SPHDEM_WARM_HIST_MAX * ns);
                K.hist_n = ns;
                K.hring = A.get<int>(2);
                K.ppart = A.get<double>((size_t)PROJ_NV * KRY_G);
                K.pc = A.get<double>(PROJ_MAX + 2);
                K.AD = A.get<double>((size_t)PROJ_MAX * ns);
                if (!A.ok) return SPHDEM_E_NOMEM;
            }
            if (p.warm_start == SPHDEM_WARM_MLP) {
                K.fraw = A.get<float>((size_t)ns * MLP_FEAT);
                K.feat = A.get<__nv_bfloat16>((size_t)ns * MLP_FEAT);
                K.pprev = A.get<double>(ns);
                K.x0 = A.get<double>(ns);
                K.yp = A.get<float>(ns);
                K.target = A.get<float>(ns);
                K.weight = A.get<float>(ns);
                K.mpart = A.get<double>((size_t)KRY_G * MPART_W);
                K.mstat = A.get<double>(MS_COUNT);
                if (!A.ok) return SPHDEM_E_NOMEM;
                if ((r = mlp_alloc(EH->net))) return r;
                if ((r = mlp_init_params(EH->net, (unsigned)p.mlp_seed, st))) return r;
                EH->has_mlp = true;
            }
        }
        CK(cudaMemsetAsync(E.flags, 0, sizeof(DevFlags), st));
        CK(cudaStreamSynchronize(st));
    }
    {
        DevFlags f0;
        std::memset(&f0, 0, sizeof(f0));
        f0.step_count = H->count;
        CK(cudaMemcpy(E.flags, &f0, sizeof(f0), cudaMemcpyHostToDevice));
    }
    if (ns > 0 && nd > 0 && !H->dem_stream) {
        CK(cudaStreamCreateWithFlags(&H->dem_stream, cudaStreamNonBlocking));
        for (cudaEvent_t& e : H->fork_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    H->committed = true;
    return SPHDEM_OK;
}

// ---------------------------------------------------------------------------
// field access
// ---------------------------------------------------------------------------
template <typename R>
static int field_ptr(SphdemHandle* H, int which, int field, const void** ptr, int* kind) {
    // kind: 0 double, 1 R, 2 int
    EngineHost<R>* EH = (EngineHost<R>*)H->eng;
    Engine<R>& E = EH->E;
    const DevParams& P = E.P;
    if (which == SPHDEM_SPH) {
        SphState<R>& S = E.S[E.cur_s];
        SphWork<R>& W = E.sw;
        bool xs = P.xsph;
        switch (field) {
        case SPHDEM_F_X: *ptr = S.x; *kind = 0; return 0;
        case SPHDEM_F_Y: *ptr = S.y; *kind = 0; return 0;
        case SPHDEM_F_Z: *ptr = S.z; *kind = 0; return 0;
        case SPHDEM_F_H: *ptr = S.h; *kind = 0; return 0;
        case SPHDEM_F_UX: *ptr = xs ? W.u_tmpx : S.ux; *kind = 1; return 0;
        case SPHDEM_F_UY: *ptr = xs ? W.u_tmpy : S.uy; *kind = 1; return 0;
        case SPHDEM_F_UZ: *ptr = xs ? W.u_tmpz : S.uz; *kind = 1; return 0;
        case SPHDEM_F_TEMP: *ptr = xs ? W.temp_tmp : S.temp; *kind = 1; return 0;
        case SPHDEM_F_M: *ptr = W.m_new; *kind = 1; return 0;
        case SPHDEM_F_RHO: *ptr = W.rho_new; *kind = 1; return 0;
        case SPHDEM_F_PRES: *ptr = W.p_new; *kind = 1; return 0;
        case SPHDEM_F_DEMPOR: *ptr = W.DEMpor; *kind = 1; return 0;
        case SPHDEM_F_DDEMPOR: *ptr = S.dDEMpor; *kind = 1; return 0;
        case SPHDEM_F_FLT_S: *ptr = S.flt_s; *kind = 1; return 0;
        case SPHDEM_F_FTOTALX: *ptr = W.ftx; *kind = 1; return 0;
        case SPHDEM_F_FTOTALY: *ptr = W.fty; *kind = 1; return 0;
        case SPHDEM_F_FTOTALZ: *ptr = W.ftz; *kind = 1; return 0;
        case SPHDEM_F_FPX: *ptr = W.fpx; *kind = 1; return 0;
        case SPHDEM_F_FPY: *ptr = W.fpy; *kind = 1; return 0;
        case SPHDEM_F_FPZ: *ptr = W.fpz; *kind = 1; return 0;
        case SPHDEM_F_PGFX: *ptr = W.pgfx; *kind = 1; return 0;
        case SPHDEM_F_PGFY: *ptr = W.pgfy; *kind = 1; return 0;
        case SPHDEM_F_PGFZ: *ptr = W.pgfz; *kind = 1; return 0;
        case SPHDEM_F_RHO_REF: *ptr = W.rho_ref; *kind = 1; return 0;
        case SPHDEM_F_DTEMP: *ptr = W.dtemp; *kind = 1; return 0;
        case SPHDEM_F_VIS_T: *ptr = W.vist; *kind = 1; return 0;
        case SPHDEM_F_PTYPE: *ptr = S.ptype; *kind = 2; return 0;
        case SPHDEM_F_ITYPE: *ptr = S.itype; *kind = 2; return 0;
        case SPHDEM_F_BUFFER_TYPE: *ptr = S.btype; *kind = 2; return 0;
        case SPHDEM_F_PID: *ptr = S.pid; *kind = 2; return 0;
        case SPHDEM_F_CELL: *ptr = W.key_out; *kind = 2; return 0;
        }
    } else {
        DemState<double>& D = E.D[E.cur_d];
        DemWork<double>& DW = E.dw;
        switch (field) {
        case SPHDEM_F_X: *ptr = D.x; *kind = 0; return 0;
        case SPHDEM_F_Y: *ptr = D.y; *kind = 0; return 0;
        case SPHDEM_F_Z: *ptr = D.z; *kind = 0; return 0;
        case SPHDEM_F_H: *ptr = D.h; *kind = 0; return 0;
        case SPHDEM_F_RAD: *ptr = D.rad; *kind = 0; return 0;
        case SPHDEM_F_UX: *ptr = D.ux; *kind = 0; return 0;
        case SPHDEM_F_UY: *ptr = D.uy; *kind = 0; return 0;
        case SPHDEM_F_UZ: *ptr = D.uz; *kind = 0; return 0;
        case SPHDEM_F_WX: *ptr = D.wx; *kind = 0; return 0;
        case SPHDEM_F_WY: *ptr = D.wy; *kind = 0; return 0;
        case SPHDEM_F_WZ: *ptr = D.wz; *kind = 0; return 0;
        case SPHDEM_F_M: *ptr = D.m; *kind = 0; return 0;
        case SPHDEM_F_RHO: *ptr = D.rho; *kind = 0; return 0;
        case SPHDEM_F_RI: *ptr = D.ri; *kind = 0; return 0;
        case SPHDEM_F_TEMP: *ptr = D.temp; *kind = 0; return 0;
        case SPHDEM_F_TEMP1: *ptr = D.temp1; *kind = 0; return 0;
        case SPHDEM_F_TEMP2: *ptr = D.temp2; *kind = 0; return 0;
        case SPHDEM_F_TEMP3: *ptr = D.temp3; *kind = 0; return 0;
        case SPHDEM_F_FDX_DF: *ptr = D.Fdx_df; *kind = 0; return 0;
        case SPHDEM_F_FDY_DF: *ptr = D.Fdy_df; *kind = 0; return 0;
        case SPHDEM_F_FDZ_DF: *ptr = D.Fdz_df; *kind = 0; return 0;
        case SPHDEM_F_Q_SD: *ptr = D.Q_sd; *kind = 0; return 0;
        case SPHDEM_F_DEMPOR: *ptr = DW.DEMpor; *kind = 0; return 0;
        case SPHDEM_F_FLT_S: *ptr = DW.flt_s; *kind = 0; return 0;
        case SPHDEM_F_FLT_SD: *ptr = DW.flt_sd; *kind = 0; return 0;
        case SPHDEM_F_FLT_SD2: *ptr = DW.flt_sd2; *kind = 0; return 0;
        case SPHDEM_F_FTOTALX: *ptr = DW.ftx; *kind = 0; return 0;
        case SPHDEM_F_FTOTALY: *ptr = DW.fty; *kind = 0; return 0;
        case SPHDEM_F_FTOTALZ: *ptr = DW.ftz; *kind = 0; return 0;
        case SPHDEM_F_TORQX: *ptr = DW.tqx; *kind = 0; return 0;
        case SPHDEM_F_TORQY: *ptr = DW.tqy; *kind = 0; return 0;
        case SPHDEM_F_TORQZ: *ptr = DW.tqz; *kind = 0; return 0;
        case SPHDEM_F_DTEMP: *ptr = DW.dtemp; *kind = 0; return 0;
        case SPHDEM_F_PTYPE: *ptr = D.ptype; *kind = 2; return 0;
        case SPHDEM_F_ITYPE: *ptr = D.itype; *kind = 2; return 0;
        case SPHDEM_F_BUFFER_TYPE: *ptr = D.btype; *kind = 2; return 0;
        case SPHDEM_F_PID: *ptr = D.pid; *kind = 2; return 0;
        case SPHDEM_F_DEM_IDX: *ptr = D.dem_idx; *kind = 2; return 0;
        case SPHDEM_F_CELL: *ptr = DW.key_out; *kind = 2; return 0;
        }
    }
    return SPHDEM_E_ARG;
}

template <typename R>
static int get_field_t(SphdemHandle* H, int which, int field, void* dst, int n) {
    const void* ptr;
    int kind;
    if (field_ptr<R>(H, which, field, &ptr, &kind)) return SPHDEM_E_ARG;
    if (n == 0) return SPHDEM_OK;
    CK(cudaStreamSynchronize(H->stream));
    if (kind == 0) {
        CK(cudaMemcpy(dst, ptr, sizeof(double) * n, cudaMemcpyDeviceToHost));
    } else if (kind == 1) {
        const DevParams& P = ((EngineHost<R>*)H->eng)->E.P;
        return download_real<R>((double*)dst, (const R*)ptr, n, H->stream, field_offset(P, which, field));
    } else {
        CK(cudaMemcpy(dst, ptr, sizeof(int) * n, cudaMemcpyDeviceToHost));
    }
    return SPHDEM_OK;
}

template <typename R>
static int stats_t(SphdemHandle* H, SphdemStats* out) {
    EngineHost<R>* EH = (EngineHost<R>*)H->eng;
    Engine<R>& E = EH->E;
    const DevParams& P = E.P;
    std::memset(out, 0, sizeof(*out));
    cudaStream_t st = H->stream;
    SphState<R>& S = E.S[E.cur_s];
    SphWork<R>& W = E.sw;
    DemState<double>& D = E.D[E.cur_d];
    double hb[8] = {0};
    if (P.ns > 0) {
        CK(cudaMemsetAsync(E.red_buf, 0, sizeof(double) * 3, st));
        k_stats<R><<<std::min(nblocks(P.ns, 256), 592), 256, 0, st>>>(P.ns, W.rho_new, P.xsph ? W.u_tmpx : S.ux, P.xsph ? W.u_tmpy : S.uy,
                                      P.xsph ? W.u_tmpz : S.uz, W.ftot, S.ptype, S.itype, E.red_buf, E.flags);
        CK(cudaMemcpyAsync(hb, E.red_buf, sizeof(double) * 3, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        out->rho_max_sph = hb[0]; out->u_max_sph = hb[1]; out->ftotal_max_sph = hb[2];
    }
    if (P.nd > 0) {
        CK(cudaMemsetAsync(E.red_buf, 0, sizeof(double) * 3, st));
        k_stats<double><<<std::min(nblocks(P.nd, 256), 592), 256, 0, st>>>(P.nd, D.rho, D.ux, D.uy, D.uz, (const double*)nullptr, D.ptype, D.itype, E.red_buf,
                                      E.flags);
        CK(cudaMemcpyAsync(hb, E.red_buf, sizeof(double) * 3, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        out->rho_max_dem = hb[0]; out->u_max_dem = hb[1]; out->ftotal_max_dem = hb[2];
    }
    DevFlags f;
    CK(cudaMemcpyAsync(&f, E.flags, sizeof(f), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    out->count = H->count;
    out->time = H->time;
    out->ppe_iters = 1;               // the reference's single sweep
    out->ppe_rel_residual = 0.0;      // not formed by the reference sweep
    if (H->p.ppe_mode != SPHDEM_PPE_REFERENCE && EH->K.sc) {
        double sc[KS_COUNT];
        CK(cudaMemcpyAsync(sc, EH->K.sc, sizeof(sc), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        out->ppe_iters = (int32_t)sc[KS_ITER];
        out->ppe_rel_residual = sc[KS_RES];
        out->ppe_status = (int32_t)sc[KS_STATUS];
        out->ppe_initial_residual = sc[KS_RES0];
        if (EH->K.pc) {
            double pc[2];
            CK(cudaMemcpy(pc, EH->K.pc + PROJ_MAX, sizeof(pc), cudaMemcpyDeviceToHost));
            out->ppe_warm_dirs = (int32_t)pc[0];
            out->ppe_warm_gain = pc[1];
        }
    }
    if (EH->has_mlp) {
        float loss[2] = {0, 0};
        CK(cudaMemcpy(loss, EH->net.loss, sizeof(loss), cudaMemcpyDeviceToHost));
        out->mlp_loss = loss[1] > 0 ? loss[0] / loss[1] : loss[0];
        out->mlp_phase = EH->mlp_trained < H->p.mlp_train_steps ? 1 : 2;
        out->mlp_trained_steps = EH->mlp_trained;
    }
    out->ppe_ms = H->ppe_ms;
    out->overflow_flags = f.overflow;
    out->nan_flag = f.nan;
    return SPHDEM_OK;
}

template <typename R>
static void destroy_t(SphdemHandle* H) {
    EngineHost<R>* EH = (EngineHost<R>*)H->eng;
    if (!EH) return;
    for (void* p : EH->A.ptrs) cudaFree(p);
    if (EH->has_mlp) mlp_free(EH->net);
    delete EH;
    H->eng = nullptr;
}

// ---------------------------------------------------------------------------
// 2-D WCSPH (solver_type WCSPH, dim 2): wcsph2d.cuh.  Its own state and
// work arrays behind the same handle (H->kind == 1).
// ---------------------------------------------------------------------------
template <typename R>
struct WEngineHost {
    DevParams P;
    WParams Q;
    WState<R> S[2];
    int cur = 0;
    WWork<R> W;
    DevFlags* flags = nullptr;
    double* red_buf = nullptr;    // maxima of sphdem_get_stats (3 doubles)
    CellSort cs;      // NNPS sort by cell
    int nb_cap = 0;
    int lanes = 1;    // lanes per particle of the gathers (w_lanes, or the commit-time autotuner)
    Alloc A;
};

// launch KERN<R, L> with L lanes per particle (n L threads in blocks of TPB)
#define W_LAUNCH(L, KERN, n, st, ...)                                                                      \
    do {                                                                                                   \
        switch (L) {                                                                                       \
        case 1: KERN<R, 1><<<nblocks((n) * 1, TPB), TPB, 0, st>>>(__VA_ARGS__); break;                    \
        case 2: KERN<R, 2><<<nblocks((n) * 2, TPB), TPB, 0, st>>>(__VA_ARGS__); break;                    \
        case 4: KERN<R, 4><<<nblocks((n) * 4, TPB), TPB, 0, st>>>(__VA_ARGS__); break;                    \
        case 8: KERN<R, 8><<<nblocks((n) * 8, TPB), TPB, 0, st>>>(__VA_ARGS__); break;                    \
        default: KERN<R, 16><<<nblocks((n) * 16, TPB), TPB, 0, st>>>(__VA_ARGS__); break;                 \
        }                                                                                                  \
    } while (0)

template <typename R>
static void w_alloc_state(Alloc& A, WState<R>& S, int n) {
    S.x = A.get<double>(n); S.y = A.get<double>(n); S.z = A.get<double>(n); S.h = A.get<double>(n);
    S.m = A.get<double>(n); S.rho = A.get<double>(n);
    S.ux = A.get<R>(n); S.uy = A.get<R>(n); S.pres = A.get<R>(n); S.temp = A.get<R>(n); S.flt_s = A.get<R>(n);
    S.x0 = A.get<double>(n); S.y0 = A.get<double>(n); S.rho0 = A.get<double>(n);
    S.ux0 = A.get<R>(n); S.uy0 = A.get<R>(n);
    S.ptype = A.get<int>(n); S.btype = A.get<int>(n); S.itype = A.get<int>(n); S.pid = A.get<int>(n);
    S.bed = nullptr;
    S.boff = nullptr;
}

// NNPS of the WCSPH state: S[src] -> S[dst] in cell order (hashed: the
// predictor already wrote the cell keys)
template <typename R>
static int w_nnps(SphdemHandle* H, WEngineHost<R>* EH, int src, int dst, bool hashed = false) {
    const DevParams& P = EH->P;
    WWork<R>& W = EH->W;
    cudaStream_t st = H->stream;
    int n = P.ns;
    WState<R>& S = EH->S[src];
    if (!hashed) k_w_hash<R><<<nblocks(n, TPB), TPB, 0, st>>>(P, S, W.key_in, EH->cs.cnt);
    CK(cell_sort(EH->cs, n, W.key_in, W.val_out, W.key_out, W.g_str, W.g_end, st));
    k_w_gather<R><<<nblocks(n, TPB), TPB, 0, st>>>(P, S, EH->S[dst], W.val_out);
    k_rows<<<nblocks(P.NI * P.NJ * P.NK, TPB), TPB, 0, st>>>(P, W.g_str, W.g_end, W.rows);
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

// one step of WCSPH_Calc.cuh:15-340 (Lagrangian variant)
template <typename R>
static int w_enqueue(SphdemHandle* H, WEngineHost<R>* EH, int64_t* nl) {
    const DevParams& P = EH->P;
    const WParams& Q = EH->Q;
    WWork<R>& W = EH->W;
    cudaStream_t st = H->stream;
    int n = P.ns, so = EH->cur, sn = 1 - EH->cur;
    int bs = nblocks(n, TPB);
    { KTIME(KT_W_PRED); k_w_predictor<R><<<bs, TPB, 0, st>>>(P, Q, EH->S[so], W, W.key_in, EH->cs.cnt); }
    {
        KTIME(KT_W_NNPS);
        int r = w_nnps<R>(H, EH, so, sn, true);
        if (r) return r;
    }
    WState<R>& S = EH->S[sn];
    const int L = EH->lanes;
    { KTIME(KT_W_LIST); W_LAUNCH(L, k_w_list, n, st, P, S, W.rows, W.nbr, W.ncnt, EH->flags); }
    // gradient_correction() runs for kgc_solve > 0 or Antuono, but only the
    // KGC case fills Cm, and only KGC reads it (apply_gradient_correction_2D)
    if (P.kgc == 1) { KTIME(KT_W_KGC); W_LAUNCH(L, k_w_kgc, n, st, P, S, W); }
    { KTIME(KT_W_PREP); W_LAUNCH(L, k_w_prep, n, st, P, Q, S, W, EH->flags); }
    { KTIME(KT_W_CONT); W_LAUNCH(L, k_w_continuity, n, st, P, Q, S, W); }   // + EOS
    { KTIME(KT_W_INTER); W_LAUNCH(L, k_w_interaction, n, st, P, Q, S, W); }
    { KTIME(KT_W_CORR); k_w_corrector<R><<<bs, TPB, 0, st>>>(P, Q, S, W, EH->flags); }
    if (P.xsph) {
        { KTIME(KT_W_XSPH); W_LAUNCH(L, k_w_xsph, n, st, P, S, W); }
        { KTIME(KT_W_FINISH); k_w_finish<R><<<bs, TPB, 0, st>>>(P, S, W); }
    }
    CK(cudaGetLastError());
    // engine kernels of the step: predictor (+ cell keys and counts), the
    // four cell-sort passes, gather, rows, list, [kgc], prep, continuity
    // (+ EOS), interaction, corrector (+ step counter), [xsph, finish]
    *nl += 12 + (P.kgc == 1) + 2 * (P.xsph != 0);
    return SPHDEM_OK;
}

template <typename R>
static int w_run_step(SphdemHandle* H, WEngineHost<R>* EH, int64_t* nl) {
    int key = (1 << 16) | EH->cur;
    int64_t n = 0;
    if (H->use_graphs) {
        auto it = H->graphs.find(key);
        if (it == H->graphs.end()) {
            cudaGraph_t g;
            if (H->timing) std::fill(H->ev_used.begin(), H->ev_used.end(), 0);
            CK(cudaStreamBeginCapture(H->stream, cudaStreamCaptureModeThreadLocal));
            H->capturing = true;
            int r = w_enqueue<R>(H, EH, &n);
            H->capturing = false;
            cudaError_t ce = cudaStreamEndCapture(H->stream, &g);
            if (r) return r;
            if (ce != cudaSuccess) return SPHDEM_E_CUDA;
            cudaGraphExec_t ge;
            CK(cudaGraphInstantiate(&ge, g, 0));
            cudaGraphDestroy(g);
            H->graphs[key] = ge;
            H->graph_launches[key] = n;
            H->graph_kused[key] = H->ev_used;
            it = H->graphs.find(key);
        }
        n = H->graph_launches[key];
        if (H->timing) H->ev_used = H->graph_kused[key];
        CK(cudaGraphLaunch(it->second, H->stream));
    } else {
        int r = w_enqueue<R>(H, EH, &n);
        if (r) return r;
    }
    *nl += n;
    EH->cur ^= 1;
    return SPHDEM_OK;
}

// Lanes per particle of the gathers.  w_lanes > 0 fixes it; 0 times the
// gather kernels (list, [kgc], prep, continuity, interaction, [xsph]) on the
// committed, cell-sorted state for L = 1, 2, 4, 8, 16 and keeps the fastest
// (the minimum of 3 repetitions after one warm-up launch each).  The work
// arrays those kernels write are cleared afterwards, so the run starts from
// the same state whatever L was chosen; L changes only the order of the
// neighbour sums inside a particle, i.e. results at the rounding level.
template <typename R>
static int w_tune_lanes(SphdemHandle* H, WEngineHost<R>* EH) {
    const DevParams& P = EH->P;
    const WParams& Q = EH->Q;
    WWork<R>& W = EH->W;
    WState<R>& S = EH->S[1];   // the sorted copy that w_nnps left there
    cudaStream_t st = H->stream;
    const int n = P.ns;
    int want = H->p.w_lanes;
    if (want != 0) {
        EH->lanes = want;
        return SPHDEM_OK;
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto pass = [&](int L) {
        W_LAUNCH(L, k_w_list, n, st, P, S, W.rows, W.nbr, W.ncnt, EH->flags);
        if (P.kgc == 1) W_LAUNCH(L, k_w_kgc, n, st, P, S, W);
        W_LAUNCH(L, k_w_prep, n, st, P, Q, S, W, EH->flags);
        W_LAUNCH(L, k_w_continuity, n, st, P, Q, S, W);
        W_LAUNCH(L, k_w_interaction, n, st, P, Q, S, W);
        if (P.xsph) W_LAUNCH(L, k_w_xsph, n, st, P, S, W);
    };
    float best = 1e30f;
    int bestL = 1;
    int rc = SPHDEM_OK;
    for (int L : {1, 2, 4, 8, 16}) {
        pass(L);
        if (cudaEventRecord(e0, st) != cudaSuccess) { rc = SPHDEM_E_CUDA; break; }
        for (int rep = 0; rep < 3; rep++) pass(L);
        float ms = 0.f;
        if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            rc = SPHDEM_E_CUDA;
            break;
        }
        if (ms < best) {
            best = ms;
            bestL = L;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    EH->lanes = bestL;
    // back to the state of a run that never tuned
    const size_t rb = sizeof(R) * (size_t)n;
    R* rz[] = {W.ftx, W.fty, W.ftot, W.drho, W.grx, W.gry, W.pgfx, W.pgfy};
    for (R* a : rz) CK(cudaMemsetAsync(a, 0, rb, st));
    CK(cudaMemsetAsync(W.Cm, 0, rb * 4, st));
    CK(cudaMemsetAsync(W.rho_ref, 0, sizeof(double) * n, st));
    CK(cudaMemsetAsync(W.xn, 0, sizeof(double) * n, st));
    CK(cudaMemsetAsync(W.yn, 0, sizeof(double) * n, st));
    CK(cudaMemsetAsync(W.ncnt, 0, sizeof(int) * n, st));
    CK(cudaStreamSynchronize(st));
    return SPHDEM_OK;
}

// Placement of a batch (sphdem_create_batch): bed b's cells are computed at
// (x + ox_b, y + oy_b), which puts the beds side by side on shelves with a
// gap of at least 8 cells (and 5 % of the bed) between beds, so that no
// stencil of one bed reaches another; positions stay as given.
static void place_batch(SphdemHandle* H, double dcell) {
    const auto& X = H->stage_d[0][SPHDEM_F_X];
    const auto& Y = H->stage_d[0][SPHDEM_F_Y];
    int nb = (int)H->bed_start.size() - 1;
    std::vector<double> x0(nb), x1(nb), y0(nb), y1(nb);
    double area = 0, wmax = 0;
    for (int b = 0; b < nb; b++) {
        int a = H->bed_start[b], e = H->bed_start[b + 1];
        x0[b] = x1[b] = X[a];
        y0[b] = y1[b] = Y[a];
        for (int k = a; k < e; k++) {
            x0[b] = std::min(x0[b], X[k]); x1[b] = std::max(x1[b], X[k]);
            y0[b] = std::min(y0[b], Y[k]); y1[b] = std::max(y1[b], Y[k]);
        }
        double g = std::max(8.0 * dcell, 0.05 * std::max(x1[b] - x0[b], y1[b] - y0[b]));
        area += (x1[b] - x0[b] + g) * (y1[b] - y0[b] + g);
        wmax = std::max(wmax, x1[b] - x0[b] + g);
    }
    double limit = std::max(wmax, std::sqrt(area));
    double cx = 0, cy = 0, shelf = 0;
    H->bed_off.assign(2 * nb, 0.0);
    for (int b = 0; b < nb; b++) {
        double g = std::max(8.0 * dcell, 0.05 * std::max(x1[b] - x0[b], y1[b] - y0[b]));
        double w = x1[b] - x0[b] + g, h = y1[b] - y0[b] + g;
        if (cx > 0 && cx + w > limit) {
            cy += shelf;
            cx = 0;
            shelf = 0;
        }
        H->bed_off[2 * b] = cx - x0[b];
        H->bed_off[2 * b + 1] = cy - y0[b];
        cx += w;
        shelf = std::max(shelf, h);
    }
}

template <typename R>
static int w_commit_t(SphdemHandle* H) {
    const SphdemParams& p = H->p;
    int ns = H->ns;
    if (!H->bed_start.empty()) {
        if (H->have_file_order) return SPHDEM_E_ARG;
        auto& hv = H->stage_d[0][SPHDEM_F_H];
        if ((int)hv.size() != ns || (int)H->stage_d[0][SPHDEM_F_X].size() != ns ||
            (int)H->stage_d[0][SPHDEM_F_Y].size() != ns)
            return SPHDEM_E_INPUT;
        double hmax = 0;
        for (double v : hv) hmax = std::max(hmax, v);
        place_batch(H, 1.1 * p.kappa * hmax);
    }
    // bounding box and grid as the ISPH engine (function_init.cuh:913-950);
    // a batch's box is that of the placed beds
    std::vector<double> fx = H->have_file_order ? H->file_x : H->stage_d[0][SPHDEM_F_X];
    std::vector<double> fy = H->have_file_order ? H->file_y : H->stage_d[0][SPHDEM_F_Y];
    for (int b = 0; b + 1 < (int)H->bed_start.size(); b++)
        for (int k = H->bed_start[b]; k < H->bed_start[b + 1]; k++) {
            fx[k] += H->bed_off[2 * b];
            fy[k] += H->bed_off[2 * b + 1];
        }
    std::vector<double> fz = H->have_file_order ? H->file_z : H->stage_d[0][SPHDEM_F_Z];
    double h0 = H->have_file_order ? H->file_h0 : H->stage_d[0][SPHDEM_F_H][0];
    int n = (int)fx.size();
    if (fz.size() != fx.size()) fz.assign(fx.size(), 0.0);
    for (double z : fz)
        if (z != fz[0]) return SPHDEM_E_INPUT;   // 2-D: one z for every particle
    double mnx = fx[0], mxx = fx[0], mny = fy[0], mxy = fy[0];
    for (int k = 0; k < n - 1; k++) {
        mnx = std::min(mnx, fx[k]); mxx = std::max(mxx, fx[k]);
        mny = std::min(mny, fy[k]); mxy = std::max(mxy, fy[k]);
    }
    mnx -= (mxx - mnx) * p.margin[0]; mxx += (mxx - mnx) * p.margin[1];
    mny -= (mxy - mny) * p.margin[2]; mxy += (mxy - mny) * p.margin[3];
    double dcell = 1.1 * p.kappa * h0;
    int NI = (int)((mxx - mnx) / dcell) + 1, NJ = (int)((mxy - mny) / dcell) + 1, NK = 1;
    if (!(dcell > 0) || (double)NI * NJ > 2.0e9) return SPHDEM_E_INPUT;
    H->bbox[0] = mnx; H->bbox[1] = mxx; H->bbox[2] = mny; H->bbox[3] = mxy; H->bbox[4] = fz[0]; H->bbox[5] = fz[0];
    H->nijk[0] = NI; H->nijk[1] = NJ; H->nijk[2] = NK;
    H->dcell = dcell;
    auto* EH = new WEngineHost<R>();
    H->eng = EH;
    H->kind = 1;
    DevParams& P = EH->P;
    std::memset(&P, 0, sizeof(P));
    P.kernel_type = p.kernel_type; P.dim = 2; P.kgc = p.kgc_solve;
    P.fp = p.fp_solve; P.fv = p.fv_solve; P.fva = p.fva_solve; P.fg = p.fg_solve; P.xsph = p.xsph_solve;
    P.NI = NI; P.NJ = NJ; P.NK = NK; P.num_cells = NI * NJ * NK + 1;
    P.ns = ns;
    P.kappa = p.kappa; P.dt = p.dt; P.sdt = p.dt; P.soundspeed = p.soundspeed; P.u_limit = p.u_limit;
    P.c_xsph = p.c_xsph;
    P.xmin = mnx; P.xmax = mxx; P.ymin = mny; P.ymax = mxy; P.zmin = fz[0]; P.zmax = fz[0];
    P.mu_gas = p.mu_gas; P.g_sph = p.g_sph;
    WParams& Q = EH->Q;
    Q.alpha = p.art_visc_alpha; Q.beta = p.art_visc_beta; Q.delta = p.delta_sph;
    Q.freq_filt = p.freq_filt; Q.delsph = p.delSPH_solve; Q.rho_cont = p.rho_type == 1;
    Q.gamma = p.gamma; Q.eos_B = p.soundspeed * p.soundspeed * 1.186 / p.gamma;
    Alloc& A = EH->A;
    w_alloc_state<R>(A, EH->S[0], ns);
    w_alloc_state<R>(A, EH->S[1], ns);
    if (!H->bed_start.empty()) {
        int nb = (int)H->bed_start.size() - 1;
        EH->S[0].bed = A.get<int>(ns);
        EH->S[1].bed = A.get<int>(ns);
        double2* boff = A.get<double2>(nb);
        if (!A.ok) return SPHDEM_E_NOMEM;
        CK(cudaMemcpy(boff, H->bed_off.data(), sizeof(double2) * nb, cudaMemcpyHostToDevice));
        std::vector<int> bed(ns);
        for (int b = 0; b < nb; b++)
            for (int k = H->bed_start[b]; k < H->bed_start[b + 1]; k++) bed[k] = b;
        CK(cudaMemcpy(EH->S[0].bed, bed.data(), sizeof(int) * ns, cudaMemcpyHostToDevice));
        EH->S[0].boff = EH->S[1].boff = boff;
    }
    WWork<R>& W = EH->W;
    W.ftx = A.get<R>(ns); W.fty = A.get<R>(ns); W.ftot = A.get<R>(ns); W.drho = A.get<R>(ns);
    W.rho_ref = A.get<double>(ns); W.grx = A.get<R>(ns); W.gry = A.get<R>(ns); W.pgfx = A.get<R>(ns);
    W.pgfy = A.get<R>(ns); W.Cm = A.get<R>((size_t)ns * 4);
    W.xn = A.get<double>(ns); W.yn = A.get<double>(ns); W.rhon = A.get<double>(ns);
    W.key_in = A.get<int>(ns); W.key_out = A.get<int>(ns); W.val_in = nullptr; W.val_out = A.get<int>(ns);
    W.g_str = A.get<int>(P.num_cells + 1); W.g_end = A.get<int>(P.num_cells + 1);
    W.rows = A.get<int4>(NI * NJ * NK);
    W.ncnt = A.get<int>(ns);
    W.nbr = nullptr;
    EH->flags = A.get<DevFlags>(1);
    EH->red_buf = A.get<double>(4);
    if (!A.ok) return SPHDEM_E_NOMEM;
    EH->cs = alloc_cell_sort(A, P.num_cells, ns);
    if (!A.ok) return SPHDEM_E_NOMEM;
    cudaStream_t st = H->stream;
    auto& pt = H->stage_i[0][SPHDEM_F_PTYPE];
    for (int v : pt)
        if (v == 9 || v > 1000) return SPHDEM_E_UNSUPPORTED;   // moving plates, DEM
    std::vector<int> itype(ns, 1), btype(ns, 0), pid(ns);
    for (int i = 0; i < ns; i++) pid[i] = i;
    H->stage_i[0][SPHDEM_F_ITYPE] = itype;
    H->stage_i[0][SPHDEM_F_BUFFER_TYPE] = btype;
    H->stage_i[0][SPHDEM_F_PID] = pid;
    WState<R>& S = EH->S[0];
    auto up_d = [&](double* dst, int f) -> int {
        auto& v = H->stage_d[0][f];
        if ((int)v.size() != ns) v.assign(ns, 0.0);
        CK(cudaMemcpy(dst, v.data(), sizeof(double) * ns, cudaMemcpyHostToDevice));
        return SPHDEM_OK;
    };
    auto up_r = [&](R* dst, int f) -> int {
        auto& v = H->stage_d[0][f];
        if ((int)v.size() != ns) v.assign(ns, 0.0);
        return upload_real<R>(dst, v.data(), ns, st);
    };
    auto up_i = [&](int* dst, int f) -> int {
        auto& v = H->stage_i[0][f];
        if ((int)v.size() != ns) v.assign(ns, 0);
        CK(cudaMemcpy(dst, v.data(), sizeof(int) * ns, cudaMemcpyHostToDevice));
        return SPHDEM_OK;
    };
    int r = 0;
    r |= up_d(S.x, SPHDEM_F_X); r |= up_d(S.y, SPHDEM_F_Y); r |= up_d(S.z, SPHDEM_F_Z); r |= up_d(S.h, SPHDEM_F_H);
    r |= up_r(S.ux, SPHDEM_F_UX); r |= up_r(S.uy, SPHDEM_F_UY); r |= up_d(S.m, SPHDEM_F_M);
    r |= up_d(S.rho, SPHDEM_F_RHO); r |= up_r(S.pres, SPHDEM_F_PRES); r |= up_r(S.temp, SPHDEM_F_TEMP);
    r |= up_r(S.flt_s, SPHDEM_F_FLT_S);
    r |= up_i(S.ptype, SPHDEM_F_PTYPE); r |= up_i(S.btype, SPHDEM_F_BUFFER_TYPE); r |= up_i(S.itype, SPHDEM_F_ITYPE);
    r |= up_i(S.pid, SPHDEM_F_PID);
    if (r) return SPHDEM_E_CUDA;
    // neighbour-list capacity from an exact count on the sorted input
    if ((r = w_nnps<R>(H, EH, 0, 1))) return r;
    k_w_list<R, 1><<<nblocks(ns, TPB), TPB, 0, st>>>(P, EH->S[1], W.rows, nullptr, W.ncnt, EH->flags);
    CK(cudaGetLastError());
    DevFlags f;
    CK(cudaMemcpyAsync(&f, EH->flags, sizeof(f), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int cap = std::max(32, ((int)(f.max_ncnt * 1.25) + 16 + 7) / 8 * 8);
    P.nb_cap = cap;
    EH->nb_cap = cap;
    W.nbr = A.get<int>((size_t)cap * ns);
    if (!A.ok) return SPHDEM_E_NOMEM;
    if ((r = w_tune_lanes<R>(H, EH))) return r;
    DevFlags f0;
    std::memset(&f0, 0, sizeof(f0));
    f0.step_count = H->count;
    CK(cudaMemcpy(EH->flags, &f0, sizeof(f0), cudaMemcpyHostToDevice));
    H->committed = true;
    return SPHDEM_OK;
}

template <typename R>
static int w_field_ptr(SphdemHandle* H, int field, const void** ptr, int* kind) {
    auto* EH = (WEngineHost<R>*)H->eng;
    WState<R>& S = EH->S[EH->cur];
    WWork<R>& W = EH->W;
    switch (field) {
    case SPHDEM_F_X: *ptr = S.x; *kind = 0; return 0;
    case SPHDEM_F_Y: *ptr = S.y; *kind = 0; return 0;
    case SPHDEM_F_Z: *ptr = S.z; *kind = 0; return 0;
    case SPHDEM_F_H: *ptr = S.h; *kind = 0; return 0;
    case SPHDEM_F_UX: *ptr = S.ux; *kind = 1; return 0;
    case SPHDEM_F_UY: *ptr = S.uy; *kind = 1; return 0;
    case SPHDEM_F_M: *ptr = S.m; *kind = 0; return 0;
    case SPHDEM_F_RHO: *ptr = S.rho; *kind = 0; return 0;
    case SPHDEM_F_PRES: *ptr = S.pres; *kind = 1; return 0;
    case SPHDEM_F_TEMP: *ptr = S.temp; *kind = 1; return 0;
    case SPHDEM_F_FLT_S: *ptr = S.flt_s; *kind = 1; return 0;
    case SPHDEM_F_FTOTALX: *ptr = W.ftx; *kind = 1; return 0;
    case SPHDEM_F_FTOTALY: *ptr = W.fty; *kind = 1; return 0;
    case SPHDEM_F_PGFX: *ptr = W.pgfx; *kind = 1; return 0;
    case SPHDEM_F_PGFY: *ptr = W.pgfy; *kind = 1; return 0;
    case SPHDEM_F_RHO_REF: *ptr = W.rho_ref; *kind = 0; return 0;
    case SPHDEM_F_FTOTAL: *ptr = W.ftot; *kind = 1; return 0;
    case SPHDEM_F_DRHO: *ptr = W.drho; *kind = 1; return 0;
    case SPHDEM_F_GRAD_RHOX: *ptr = W.grx; *kind = 1; return 0;
    case SPHDEM_F_GRAD_RHOY: *ptr = W.gry; *kind = 1; return 0;
    case SPHDEM_F_PTYPE: *ptr = S.ptype; *kind = 2; return 0;
    case SPHDEM_F_ITYPE: *ptr = S.itype; *kind = 2; return 0;
    case SPHDEM_F_BUFFER_TYPE: *ptr = S.btype; *kind = 2; return 0;
    case SPHDEM_F_PID: *ptr = S.pid; *kind = 2; return 0;
    case SPHDEM_F_CELL: *ptr = W.key_out; *kind = 2; return 0;
    }
    return -1;
}

template <typename R>
static int w_get_field_t(SphdemHandle* H, int field, void* dst, int n) {
    const void* ptr;
    int kind;
    if (w_field_ptr<R>(H, field, &ptr, &kind)) return SPHDEM_E_ARG;
    if (n == 0) return SPHDEM_OK;
    CK(cudaStreamSynchronize(H->stream));
    if (kind == 0) CK(cudaMemcpy(dst, ptr, sizeof(double) * n, cudaMemcpyDeviceToHost));
    else if (kind == 1) return download_real<R>((double*)dst, (const R*)ptr, n, H->stream);
    else CK(cudaMemcpy(dst, ptr, sizeof(int) * n, cudaMemcpyDeviceToHost));
    return SPHDEM_OK;
}

template <typename R>
static int w_stats_t(SphdemHandle* H, SphdemStats* out) {
    auto* EH = (WEngineHost<R>*)H->eng;
    std::memset(out, 0, sizeof(*out));
    cudaStream_t st = H->stream;
    WState<R>& S = EH->S[EH->cur];
    double* buf = EH->red_buf;
    CK(cudaMemsetAsync(buf, 0, sizeof(double) * 3, st));
    k_stats<R, double><<<std::min(nblocks(EH->P.ns, 256), 592), 256, 0, st>>>(EH->P.ns, S.rho, S.ux, S.uy, nullptr, EH->W.ftot,
                                                                     S.ptype, S.itype, buf, EH->flags);
    double hb[3];
    CK(cudaMemcpyAsync(hb, buf, sizeof(hb), cudaMemcpyDeviceToHost, st));
    DevFlags f;
    CK(cudaMemcpyAsync(&f, EH->flags, sizeof(f), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    out->rho_max_sph = hb[0];
    out->u_max_sph = hb[1];
    out->ftotal_max_sph = hb[2];
    out->count = H->count;
    out->time = H->time;
    out->ppe_iters = 0;
    out->overflow_flags = f.overflow;
    out->nan_flag = f.nan;
    out->w_lanes = EH->lanes;
    return SPHDEM_OK;
}

template <typename R>
static void w_destroy_t(SphdemHandle* H) {
    auto* EH = (WEngineHost<R>*)H->eng;
    if (!EH) return;
    for (void* q : EH->A.ptrs) cudaFree(q);
    delete EH;
    H->eng = nullptr;
}

static void engine_destroy(SphdemHandle* h) {
    if (h->kind == 1) {
        if (h->prec == SPHDEM_PREC_FP64) w_destroy_t<double>(h); else w_destroy_t<float>(h);
    } else {
        if (h->prec == SPHDEM_PREC_FP64) destroy_t<double>(h); else destroy_t<float>(h);
    }
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
static bool is_real_field(int f) { return f >= SPHDEM_F_X && f <= SPHDEM_F_VIS_T; }
static bool is_int_field(int f) { return f >= SPHDEM_F_PTYPE && f <= SPHDEM_F_CELL; }

static int check_supported(const SphdemParams* p) {
    if (p->solver_type == SPHDEM_WCSPH) {
        // 2-D WCSPH (SOPHIA_single, WCSPH_Calc.cuh:15-340), Lagrangian variant
        if (p->dim != 2) return SPHDEM_E_UNSUPPORTED;
        if (p->prop_table || p->fs_solve || p->fb_solve || p->interface_solve || p->boussinesq_solve ||
            p->concn_solve || p->pst_solve || p->turbulence_model != 0 || p->penetration_solve || p->noslip_bc ||
            p->con_solve || p->open_boundary || p->switch_ptype)
            return SPHDEM_E_UNSUPPORTED;
        if (p->kgc_solve != 0 && p->kgc_solve != 1) return SPHDEM_E_UNSUPPORTED;
        if (p->time_type != 1 || p->rho_type != 1) return SPHDEM_E_UNSUPPORTED;   // predictor-corrector, continuity
        if (p->delSPH_solve < 0 || p->delSPH_solve > 2) return SPHDEM_E_UNSUPPORTED;
        if (p->ppe_mode != SPHDEM_PPE_REFERENCE || p->warm_start != SPHDEM_WARM_PREVIOUS) return SPHDEM_E_ARG;
        if (p->kernel_type < 0 || p->kernel_type > 5) return SPHDEM_E_ARG;
        if (!(p->dt > 0) || !(p->kappa > 0) || p->freq_filt <= 0 || !(p->gamma > 0)) return SPHDEM_E_ARG;
        if (p->w_lanes != 0 && p->w_lanes != 1 && p->w_lanes != 2 && p->w_lanes != 4 && p->w_lanes != 8 &&
            p->w_lanes != 16)
            return SPHDEM_E_ARG;
        return SPHDEM_OK;
    }
    if (p->solver_type != SPHDEM_ISPH) return SPHDEM_E_UNSUPPORTED;
    // dim 2: a bed in a plane y = const (the step's 2-D model, step_kernels.cuh)
    if (p->dim != 3 && p->dim != 2) return SPHDEM_E_UNSUPPORTED;
    // Switches of the ISPH step that are not built: property tables, the
    // Boussinesq term (functions_PPE2.cuh:1575 reads temp0, a local that is
    // never assigned), and the wall velocity condition of noslip_bc /
    // penetration_solve (ISPH_Calc_seperate.cuh:189-193 runs it on the
    // combined-mode arrays dev_SP1 / g_str, which this step never fills).
    // Accepted with their reference effect: the SPS eddy viscosity and the
    // inter-particle surface tension (pass B); other turbulence models (no
    // eddy viscosity), the curvature surface tension (its colour function is
    // never formed, so the force is zero), concentration diffusion (zero
    // diffusion coefficient, functions_PROP.cuh:460-466, and no update of
    // concn) and particle shifting (no kernel of this step reads it).
    if (p->prop_table || p->boussinesq_solve || p->penetration_solve || p->noslip_bc)
        return SPHDEM_E_UNSUPPORTED;
    if (p->turbulence_model < 0 || p->turbulence_model > 4) return SPHDEM_E_ARG;
    if (p->kgc_solve != 0 && p->kgc_solve != 1) return SPHDEM_E_UNSUPPORTED;
    if (p->time_type != 1) return SPHDEM_E_UNSUPPORTED;
    if (p->decouple_stride != 1) return SPHDEM_E_UNSUPPORTED;
    if (p->flag_z_index) return SPHDEM_E_UNSUPPORTED;
    if (p->open_boundary == 2) return SPHDEM_E_UNSUPPORTED;
    if (p->ppe_mode != SPHDEM_PPE_REFERENCE && p->ppe_mode != SPHDEM_PPE_KRYLOV && p->ppe_mode != SPHDEM_PPE_PCG)
        return SPHDEM_E_UNSUPPORTED;
    if (p->ppe_mode != SPHDEM_PPE_REFERENCE && !(p->ppe_tol > 0)) return SPHDEM_E_ARG;
    // the reference sweep always starts from the previous pressure
    if (p->warm_start == SPHDEM_WARM_MLP && p->ppe_mode == SPHDEM_PPE_REFERENCE) return SPHDEM_E_UNSUPPORTED;
    if (p->warm_start == SPHDEM_WARM_PROJECT && p->ppe_mode == SPHDEM_PPE_REFERENCE) return SPHDEM_E_UNSUPPORTED;
    if (p->warm_hist < 0 || p->warm_hist > SPHDEM_WARM_HIST_MAX) return SPHDEM_E_ARG;
    if (p->warm_fit & ~(SPHDEM_FIT_RESIDUAL | SPHDEM_FIT_AFFINE)) return SPHDEM_E_ARG;
    if (p->dem_list_cap < 0 || p->dem_list_cap > 4096) return SPHDEM_E_ARG;
    if (p->ppe_precond != SPHDEM_PRECOND_JACOBI && p->ppe_precond != SPHDEM_PRECOND_TWO_LEVEL) return SPHDEM_E_ARG;
    if (p->ppe_precond == SPHDEM_PRECOND_TWO_LEVEL && p->ppe_mode != SPHDEM_PPE_PCG) return SPHDEM_E_UNSUPPORTED;
    if (p->warm_start != SPHDEM_WARM_PREVIOUS && p->warm_start != SPHDEM_WARM_MLP &&
        p->warm_start != SPHDEM_WARM_EXTRAPOLATE && p->warm_start != SPHDEM_WARM_PROJECT)
        return SPHDEM_E_ARG;
    if (p->warm_start == SPHDEM_WARM_EXTRAPOLATE && p->ppe_mode == SPHDEM_PPE_REFERENCE) return SPHDEM_E_UNSUPPORTED;
    if (p->kernel_type < 0 || p->kernel_type > 5) return SPHDEM_E_ARG;
    if (!(p->dt > 0) || !(p->kappa > 0) || p->freq_filt <= 0) return SPHDEM_E_ARG;
    return SPHDEM_OK;
}

extern "C" int sphdem_create(const SphdemParams* p, int32_t n_sph, int32_t n_dem, SphdemHandle** out) {
    if (!p || !out || n_sph < 0 || n_dem < 0 || n_sph + n_dem == 0) return SPHDEM_E_ARG;
    *out = nullptr;
    int r = check_supported(p);
    if (r) return r;
    if (p->solver_type == SPHDEM_WCSPH && (n_dem != 0 || n_sph == 0)) return SPHDEM_E_UNSUPPORTED;
    SphdemHandle* h = new SphdemHandle();
    h->p = *p;
    h->ns = n_sph;
    h->nd = n_dem;
    h->prec = p->precision == SPHDEM_PREC_FP64 ? SPHDEM_PREC_FP64 : SPHDEM_PREC_FP32;
    h->time = p->time;
    h->count = (int)std::floor(p->time / p->dt + 0.5);  // ISPH_Calc_seperate.cuh:522
    if (cudaGetDevice(&h->device) != cudaSuccess || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return SPHDEM_E_CUDA;
    }
    *out = h;
    return SPHDEM_OK;
}

extern "C" int sphdem_create_from_dir(const char* dir, const SphdemParams* ov, SphdemHandle** out) {
    if (!dir || !out) return SPHDEM_E_ARG;
    *out = nullptr;
    SphdemParams p;
    sphdem_io_params_default(&p);
    std::string d(dir);
    int r = sphdem_read_solv((d + "/solv.txt").c_str(), &p);
    if (r) return r;
    if (ov) {
        p.precision = ov->precision;
        p.ppe_mode = ov->ppe_mode;
        p.warm_start = ov->warm_start;
        p.ppe_tol = ov->ppe_tol;
        p.ppe_max_iter = ov->ppe_max_iter;
        p.warm_hist = ov->warm_hist;
        p.warm_fit = ov->warm_fit;
        p.w_lanes = ov->w_lanes;
        p.dem_list_cap = ov->dem_list_cap;
        p.ppe_precond = ov->ppe_precond;
        p.mlp_train_steps = ov->mlp_train_steps;
        p.mlp_updates = ov->mlp_updates;
        p.mlp_seed = ov->mlp_seed;
        p.mlp_lr = ov->mlp_lr;
    }
    if ((r = sphdem_io_check_table((d + "/data.txt").c_str()))) return r;
    SphdemHandle tmp;
    if ((r = sphdem_io_read_input_txt((d + "/input.txt").c_str(), &tmp, &p))) return r;
    SphdemHandle* h = nullptr;
    if ((r = sphdem_create(&p, tmp.ns, tmp.nd, &h))) return r;
    h->stage_d[0] = tmp.stage_d[0]; h->stage_d[1] = tmp.stage_d[1];
    h->stage_i[0] = tmp.stage_i[0]; h->stage_i[1] = tmp.stage_i[1];
    h->file_x = tmp.file_x; h->file_y = tmp.file_y; h->file_z = tmp.file_z;
    h->file_h0 = tmp.file_h0;
    h->have_file_order = true;
    if ((r = sphdem_commit_particles(h))) {
        sphdem_destroy(h);
        return r;
    }
    *out = h;
    return SPHDEM_OK;
}

template <typename R>
static int set_state_t(SphdemHandle* H, int which, int field, const void* src, int n) {
    static const int allowed[] = {SPHDEM_F_X, SPHDEM_F_Y, SPHDEM_F_Z, SPHDEM_F_UX, SPHDEM_F_UY, SPHDEM_F_UZ,
                                  SPHDEM_F_WX, SPHDEM_F_WY, SPHDEM_F_WZ, SPHDEM_F_M, SPHDEM_F_RHO, SPHDEM_F_PRES,
                                  SPHDEM_F_TEMP, SPHDEM_F_DDEMPOR, SPHDEM_F_FLT_S, SPHDEM_F_FDX_DF, SPHDEM_F_FDY_DF,
                                  SPHDEM_F_FDZ_DF, SPHDEM_F_Q_SD, SPHDEM_F_TEMP1, SPHDEM_F_TEMP2, SPHDEM_F_TEMP3};
    bool ok = false;
    for (int f : allowed) ok |= (f == field);
    if (!ok) return SPHDEM_E_ARG;
    const void* ptr;
    int kind;
    if (field_ptr<R>(H, which, field, &ptr, &kind)) return SPHDEM_E_ARG;
    if (n == 0) return SPHDEM_OK;
    CK(cudaStreamSynchronize(H->stream));
    if (kind == 0) {
        CK(cudaMemcpy((void*)ptr, src, sizeof(double) * n, cudaMemcpyHostToDevice));
        return SPHDEM_OK;
    }
    const DevParams& P = ((EngineHost<R>*)H->eng)->E.P;
    return upload_real<R>((R*)ptr, (const double*)src, n, H->stream, field_offset(P, which, field));
}

// ---------------------------------------------------------------------------
// bulk field transfer: raw doubles cross the host link into (or out of) one
// device staging buffer, and one kernel converts between the staging
// buffer and the engine's fields; one stream synchronisation per call.
// ---------------------------------------------------------------------------
namespace {
struct XTab {
    void* p[SPHDEM_BULK_MAX_FIELDS];
    double off[SPHDEM_BULK_MAX_FIELDS];   // stored value = value - off (field_offset)
    unsigned dbl;   // bit f set: field f is stored as double
};

template <typename R>
__global__ void k_unstage(int n, int nf, const double* __restrict__ st, XTab t) {
    long long tot = (long long)n * nf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        int f = (int)(q / n), i = (int)(q - (long long)f * n);
        double v = st[q];
        if ((t.dbl >> f) & 1u) ((double*)t.p[f])[i] = v;
        else ((R*)t.p[f])[i] = (R)(v - t.off[f]);
    }
}

template <typename R>
__global__ void k_stage(int n, int nf, double* __restrict__ st, XTab t) {
    long long tot = (long long)n * nf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        int f = (int)(q / n), i = (int)(q - (long long)f * n);
        st[q] = ((t.dbl >> f) & 1u) ? ((const double*)t.p[f])[i] : (double)((const R*)t.p[f])[i] + t.off[f];
    }
}

// The same conversions reading / writing the caller's page-locked host
// arrays directly (mapped, through their device addresses): one kernel per
// transfer instead of a copy per field, at the link's bandwidth.
struct HTab {
    double* h[SPHDEM_BULK_MAX_FIELDS];
};

template <typename R>
__global__ void k_unstage_mapped(int n, int nf, HTab src, XTab t) {
    long long tot = (long long)n * nf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        int f = (int)(q / n), i = (int)(q - (long long)f * n);
        double v = src.h[f][i];
        if ((t.dbl >> f) & 1u) ((double*)t.p[f])[i] = v;
        else ((R*)t.p[f])[i] = (R)(v - t.off[f]);
    }
}

template <typename R>
__global__ void k_stage_mapped(int n, int nf, HTab dst, XTab t) {
    long long tot = (long long)n * nf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        int f = (int)(q / n), i = (int)(q - (long long)f * n);
        dst.h[f][i] = ((t.dbl >> f) & 1u) ? ((const double*)t.p[f])[i] : (double)((const R*)t.p[f])[i] + t.off[f];
    }
}
}  // namespace

// device address of a page-locked, mapped host range (nullptr for pageable
// memory, which then goes through cudaMemcpyAsync)
static void* mapped_host(const void* p, size_t bytes) {
    if (!p || bytes == 0) return nullptr;
    cudaPointerAttributes a, b;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || cudaPointerGetAttributes(&b, (const char*)p + bytes - 1) !=
                                                              cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || b.type != cudaMemoryTypeHost || !a.devicePointer || !b.devicePointer)
        return nullptr;
    if ((const char*)b.devicePointer - (const char*)a.devicePointer != (ptrdiff_t)(bytes - 1)) return nullptr;
    return a.devicePointer;
}

static int ensure_xfer(SphdemHandle* H, size_t elems) {
    if (elems <= H->xfer_elems) return SPHDEM_OK;
    if (H->xfer) CK(cudaFree(H->xfer));
    H->xfer = nullptr;
    H->xfer_elems = 0;
    if (cudaMalloc(&H->xfer, sizeof(double) * elems) != cudaSuccess) return SPHDEM_E_NOMEM;
    H->xfer_elems = elems;
    return SPHDEM_OK;
}

static bool is_settable_state(int f) {
    static const int allowed[] = {SPHDEM_F_X, SPHDEM_F_Y, SPHDEM_F_Z, SPHDEM_F_UX, SPHDEM_F_UY, SPHDEM_F_UZ,
                                  SPHDEM_F_WX, SPHDEM_F_WY, SPHDEM_F_WZ, SPHDEM_F_M, SPHDEM_F_RHO, SPHDEM_F_PRES,
                                  SPHDEM_F_TEMP, SPHDEM_F_DDEMPOR, SPHDEM_F_FLT_S, SPHDEM_F_FDX_DF, SPHDEM_F_FDY_DF,
                                  SPHDEM_F_FDZ_DF, SPHDEM_F_Q_SD, SPHDEM_F_TEMP1, SPHDEM_F_TEMP2, SPHDEM_F_TEMP3};
    for (int a : allowed)
        if (a == f) return true;
    return false;
}

// state of the 2-D WCSPH step that a caller may replace between steps: the
// particle fields and the last step's rates, which the next predictor reads
static bool is_settable_wcsph(int f) {
    static const int allowed[] = {SPHDEM_F_X, SPHDEM_F_Y, SPHDEM_F_UX, SPHDEM_F_UY, SPHDEM_F_M, SPHDEM_F_RHO,
                                  SPHDEM_F_PRES, SPHDEM_F_TEMP, SPHDEM_F_FLT_S, SPHDEM_F_FTOTALX, SPHDEM_F_FTOTALY,
                                  SPHDEM_F_DRHO};
    for (int a : allowed)
        if (a == f) return true;
    return false;
}

template <typename R>
static int bulk_t(SphdemHandle* H, int which, int nf, const int32_t* fields, void* const* host, bool set) {
    int n = which ? H->nd : H->ns;
    const bool w = H->kind == 1;
    if (w && which != 0) return SPHDEM_E_ARG;
    XTab t;
    t.dbl = 0;
    for (int k = 0; k < nf; k++) {
        if (!host[k]) return SPHDEM_E_ARG;
        bool ok = set ? (w ? is_settable_wcsph(fields[k]) : is_settable_state(fields[k])) : is_real_field(fields[k]);
        if (!ok) return SPHDEM_E_ARG;
        const void* ptr;
        int kind;
        int e = w ? w_field_ptr<R>(H, fields[k], &ptr, &kind) : field_ptr<R>(H, which, fields[k], &ptr, &kind);
        if (e || kind == 2) return SPHDEM_E_ARG;
        t.p[k] = (void*)ptr;
        t.off[k] = w ? 0.0 : field_offset(((EngineHost<R>*)H->eng)->E.P, which, fields[k]);
        if (kind == 0) t.dbl |= 1u << k;
    }
    if (n == 0 || nf == 0) return SPHDEM_OK;
    size_t need = (size_t)n * nf;
    cudaStream_t st = H->stream;
    int blocks = (int)std::min<long long>(((long long)need + 255) / 256, 148 * 8);
    HTab hm;
    bool mapped = true;
    for (int k = 0; k < nf && mapped; k++) {
        hm.h[k] = (double*)mapped_host(host[k], sizeof(double) * (size_t)n);
        mapped = hm.h[k] != nullptr;
    }
    if (mapped) {
        if (set) k_unstage_mapped<R><<<blocks, 256, 0, st>>>(n, nf, hm, t);
        else k_stage_mapped<R><<<blocks, 256, 0, st>>>(n, nf, hm, t);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        return SPHDEM_OK;
    }
    int r = ensure_xfer(H, need);
    if (r) return r;
    if (set) {
        for (int k = 0; k < nf; k++)
            CK(cudaMemcpyAsync(H->xfer + (size_t)k * n, host[k], sizeof(double) * n, cudaMemcpyHostToDevice, st));
        k_unstage<R><<<blocks, 256, 0, st>>>(n, nf, H->xfer, t);
        CK(cudaGetLastError());
    } else {
        k_stage<R><<<blocks, 256, 0, st>>>(n, nf, H->xfer, t);
        CK(cudaGetLastError());
        for (int k = 0; k < nf; k++)
            CK(cudaMemcpyAsync(host[k], H->xfer + (size_t)k * n, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return SPHDEM_OK;
}

extern "C" int sphdem_create_batch(const SphdemParams* p, int32_t nbeds, const int32_t* n_per_bed,
                                   SphdemHandle** out) {
    if (!p || !out || !n_per_bed || nbeds <= 0) return SPHDEM_E_ARG;
    *out = nullptr;
    if (p->solver_type != SPHDEM_WCSPH || p->dim != 2) return SPHDEM_E_UNSUPPORTED;
    std::vector<int> start(nbeds + 1, 0);
    long long tot = 0;
    for (int b = 0; b < nbeds; b++) {
        if (n_per_bed[b] <= 0) return SPHDEM_E_ARG;
        tot += n_per_bed[b];
        if (tot > (1ll << 30)) return SPHDEM_E_NOMEM;
        start[b + 1] = (int)tot;
    }
    int r = sphdem_create(p, (int32_t)tot, 0, out);
    if (r) return r;
    (*out)->bed_start = start;
    return SPHDEM_OK;
}

extern "C" int sphdem_batch_offsets(SphdemHandle* h, double* offsets) {
    if (!h || !offsets || h->bed_start.empty()) return SPHDEM_E_ARG;
    if (!h->committed) return SPHDEM_E_ARG;
    std::memcpy(offsets, h->bed_off.data(), sizeof(double) * h->bed_off.size());
    return SPHDEM_OK;
}

extern "C" int sphdem_set_fields(SphdemHandle* h, int which, int32_t nfields, const int32_t* fields,
                                 const double* const* host_src) {
    if (!h || !h->committed || !fields || !host_src || (which != 0 && which != 1) || nfields < 0 ||
        nfields > SPHDEM_BULK_MAX_FIELDS)
        return SPHDEM_E_ARG;
    return h->prec == SPHDEM_PREC_FP64
               ? bulk_t<double>(h, which, nfields, fields, (void* const*)host_src, true)
               : bulk_t<float>(h, which, nfields, fields, (void* const*)host_src, true);
}

extern "C" int sphdem_get_fields(SphdemHandle* h, int which, int32_t nfields, const int32_t* fields,
                                 double* const* host_dst) {
    if (!h || !h->committed || !fields || !host_dst || (which != 0 && which != 1) || nfields < 0 ||
        nfields > SPHDEM_BULK_MAX_FIELDS)
        return SPHDEM_E_ARG;
    return h->prec == SPHDEM_PREC_FP64
               ? bulk_t<double>(h, which, nfields, fields, (void* const*)host_dst, false)
               : bulk_t<float>(h, which, nfields, fields, (void* const*)host_dst, false);
}

extern "C" int sphdem_set_field(SphdemHandle* h, int which, int field, const void* src, size_t bytes) {
    if (!h || !src || (which != 0 && which != 1)) return SPHDEM_E_ARG;
    if (h->committed) {
        int n = which ? h->nd : h->ns;
        if (h->kind == 1) {   // 2-D WCSPH: through the bulk path
            if (!is_real_field(field) || bytes != sizeof(double) * (size_t)n) return SPHDEM_E_ARG;
            int32_t f = field;
            const double* s = (const double*)src;
            return sphdem_set_fields(h, which, 1, &f, &s);
        }
        if (!is_real_field(field) || bytes != sizeof(double) * (size_t)n) return SPHDEM_E_ARG;
        return h->prec == SPHDEM_PREC_FP64 ? set_state_t<double>(h, which, field, src, n)
                                           : set_state_t<float>(h, which, field, src, n);
    }
    int n = which ? h->nd : h->ns;
    if (is_real_field(field)) {
        if (bytes != sizeof(double) * (size_t)n) return SPHDEM_E_ARG;
        const double* s = (const double*)src;
        h->stage_d[which][field].assign(s, s + n);
        return SPHDEM_OK;
    }
    // i_type, buffer type and id are derived at commit; a slab of a larger
    // bed (sphdem_set_domain) passes its ids and parked slots (i_type 3)
    const bool slab_field = h->dom_set && (field == SPHDEM_F_PID || field == SPHDEM_F_ITYPE);
    if (is_int_field(field) && field != SPHDEM_F_CELL &&
        (slab_field || (field != SPHDEM_F_PID && field != SPHDEM_F_ITYPE && field != SPHDEM_F_BUFFER_TYPE))) {
        if (bytes != sizeof(int) * (size_t)n) return SPHDEM_E_ARG;
        const int* s = (const int*)src;
        h->stage_i[which][field].assign(s, s + n);
        return SPHDEM_OK;
    }
    return SPHDEM_E_ARG;
}

extern "C" int sphdem_commit_particles(SphdemHandle* h) {
    if (!h || h->committed) return SPHDEM_E_ARG;
    for (int q = 0; q < 2; q++) {
        int nq = q ? h->nd : h->ns;
        if (nq == 0) continue;
        for (int f : {SPHDEM_F_X, SPHDEM_F_Y, SPHDEM_F_Z, SPHDEM_F_H})
            if ((int)h->stage_d[q][f].size() != nq) return SPHDEM_E_INPUT;
        if ((int)h->stage_i[q][SPHDEM_F_PTYPE].size() != nq) return SPHDEM_E_INPUT;
        for (int i = 0; i < nq; i++) {
            int pt = h->stage_i[q][SPHDEM_F_PTYPE][i];
            if ((q == 0 && pt > 1000) || (q == 1 && pt <= 1000)) return SPHDEM_E_INPUT;
            if (!(h->stage_d[q][SPHDEM_F_H][i] > 0)) return SPHDEM_E_INPUT;
        }
        if (q == 1) {
            if ((int)h->stage_d[1][SPHDEM_F_RAD].size() != nq) return SPHDEM_E_INPUT;
            if ((int)h->stage_i[1][SPHDEM_F_DEM_IDX].size() != nq) return SPHDEM_E_INPUT;
        }
    }
    if (cudaSetDevice(h->device) != cudaSuccess) return SPHDEM_E_CUDA;
    const bool w = h->p.solver_type == SPHDEM_WCSPH;
    int r = w ? (h->prec == SPHDEM_PREC_FP64 ? w_commit_t<double>(h) : w_commit_t<float>(h))
              : (h->prec == SPHDEM_PREC_FP64 ? commit_t<double>(h) : commit_t<float>(h));
    if (r) {
        if (h->eng) engine_destroy(h);
        return r;
    }
    for (int q = 0; q < 2; q++) { h->stage_d[q].clear(); h->stage_i[q].clear(); }
    return SPHDEM_OK;
}

extern "C" int sphdem_step(SphdemHandle* h, int32_t nsteps) {
    if (!h || !h->committed || nsteps < 0) return SPHDEM_E_ARG;
    int64_t nl = 0;
    for (int k = 0; k < nsteps; k++) {
        int r;
        if (h->kind == 1)
            r = h->prec == SPHDEM_PREC_FP64 ? w_run_step<double>(h, (WEngineHost<double>*)h->eng, &nl)
                                            : w_run_step<float>(h, (WEngineHost<float>*)h->eng, &nl);
        else
            r = h->prec == SPHDEM_PREC_FP64 ? run_step<double>(h, (EngineHost<double>*)h->eng, &nl)
                                            : run_step<float>(h, (EngineHost<float>*)h->eng, &nl);
        if (r) return r;
        h->time += h->p.dt;   // ISPH_Calc_seperate.cuh:924-925
        h->count++;
    }
    h->last_launches = nl;
    return SPHDEM_OK;
}

extern "C" int sphdem_get_field(SphdemHandle* h, int which, int field, void* dst, size_t bytes) {
    if (!h || !dst || (which != 0 && which != 1)) return SPHDEM_E_ARG;
    int n = which ? h->nd : h->ns;
    if (!h->committed) {
        if (is_real_field(field)) {
            auto it = h->stage_d[which].find(field);
            if (it == h->stage_d[which].end() || bytes != sizeof(double) * (size_t)n) return SPHDEM_E_ARG;
            std::memcpy(dst, it->second.data(), bytes);
            return SPHDEM_OK;
        }
        return SPHDEM_E_ARG;
    }
    size_t need = (is_int_field(field) ? sizeof(int) : sizeof(double)) * (size_t)n;
    if (bytes != need) return SPHDEM_E_ARG;
    if (h->kind == 1) {
        if (which) return SPHDEM_E_ARG;
        return h->prec == SPHDEM_PREC_FP64 ? w_get_field_t<double>(h, field, dst, n)
                                           : w_get_field_t<float>(h, field, dst, n);
    }
    return h->prec == SPHDEM_PREC_FP64 ? get_field_t<double>(h, which, field, dst, n)
                                       : get_field_t<float>(h, which, field, dst, n);
}

extern "C" int sphdem_get_stats(SphdemHandle* h, SphdemStats* out) {
    if (!h || !out || !h->committed) return SPHDEM_E_ARG;
    if (h->kind == 1) return h->prec == SPHDEM_PREC_FP64 ? w_stats_t<double>(h, out) : w_stats_t<float>(h, out);
    return h->prec == SPHDEM_PREC_FP64 ? stats_t<double>(h, out) : stats_t<float>(h, out);
}

extern "C" int sphdem_check(SphdemHandle* h) {
    SphdemStats st;
    int r = sphdem_get_stats(h, &st);   // runs the non-finite scans, reads the status words
    if (r) return r;
    if (st.overflow_flags) return SPHDEM_E_OVERFLOW;
    if (st.nan_flag) return SPHDEM_E_NAN;
    return SPHDEM_OK;
}

extern "C" int sphdem_get_neighbors(SphdemHandle* h, int32_t* counts, int32_t* dst, int32_t cap) {
    if (!h || !counts || !h->committed || cap < 0) return SPHDEM_E_ARG;
    int ns = h->ns;
    const int* ncnt;
    const int* nbr;
    int ncap;
    if (h->kind == 1) {
        if (h->prec == SPHDEM_PREC_FP64) {
            auto* EH = (WEngineHost<double>*)h->eng;
            ncnt = EH->W.ncnt; nbr = EH->W.nbr; ncap = EH->nb_cap;
        } else {
            auto* EH = (WEngineHost<float>*)h->eng;
            ncnt = EH->W.ncnt; nbr = EH->W.nbr; ncap = EH->nb_cap;
        }
    } else if (h->prec == SPHDEM_PREC_FP64) {
        auto* EH = (EngineHost<double>*)h->eng;
        ncnt = EH->E.sw.ncnt; nbr = EH->E.sw.nbr; ncap = EH->nb_cap;
    } else {
        auto* EH = (EngineHost<float>*)h->eng;
        ncnt = EH->E.sw.ncnt; nbr = EH->E.sw.nbr; ncap = EH->nb_cap;
    }
    if (ns == 0) return SPHDEM_OK;
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(counts, ncnt, sizeof(int) * ns, cudaMemcpyDeviceToHost));
    if (!dst || cap == 0) return SPHDEM_OK;
    std::vector<int> dev((size_t)ncap * ns);
    CK(cudaMemcpy(dev.data(), nbr, sizeof(int) * dev.size(), cudaMemcpyDeviceToHost));
    // the 2-D WCSPH list is column-major, the ISPH-DEM list in blocks of 8
    // entries per particle (nb_at)
    for (int i = 0; i < ns; i++) {
        int c = std::min(std::min(counts[i], cap), ncap);
        for (int k = 0; k < c; k++)
            dst[(size_t)i * cap + k] = h->kind == 1 ? dev[(size_t)k * ns + i] : dev[nb_at(k, ns, i)];
    }
    return SPHDEM_OK;
}

// history planes (slot-major on the device) <-> particle-major host
// arrays: the transpose runs on the GPU into the bulk staging buffer, and
// the host link sees two contiguous copies.
__global__ void k_hist_out(int n, const int* __restrict__ hid, const double* __restrict__ hds, int* ids,
                           double* sp) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * SPHDEM_NSLOT) return;
    int i = q / SPHDEM_NSLOT, s = q - i * SPHDEM_NSLOT;
    ids[q] = hid[(size_t)s * n + i];
    for (int c = 0; c < 3; c++) sp[(size_t)q * 3 + c] = hds[(size_t)(s * 3 + c) * n + i];
}
__global__ void k_hist_in(int n, const int* __restrict__ ids, const double* __restrict__ sp, int* hid, double* hds) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * SPHDEM_NSLOT) return;
    int i = q / SPHDEM_NSLOT, s = q - i * SPHDEM_NSLOT;
    hid[(size_t)s * n + i] = ids[q];
    for (int c = 0; c < 3; c++) hds[(size_t)(s * 3 + c) * n + i] = sp[(size_t)q * 3 + c];
}

template <typename R>
static int history_t(SphdemHandle* H, int32_t* ids, double* sp, bool set) {
    EngineHost<R>* EH = (EngineHost<R>*)H->eng;
    DemState<double>& D = EH->E.D[EH->E.cur_d];
    int n = H->nd;
    if (n == 0) return SPHDEM_OK;
    size_t m = (size_t)n * SPHDEM_NSLOT;
    cudaStream_t st = H->stream;
    int blocks = (int)((m + 255) / 256);
    // page-locked host arrays are read in place on the way in; on the way
    // out the slot-major planes are gathered on the device first (the
    // interleaved writes of a gather straight into host memory cross the
    // link at a fraction of its bandwidth: 1.2 ms against 0.2 ms here)
    int* mid = set ? (int*)mapped_host(ids, sizeof(int) * m) : nullptr;
    double* msp = set ? (double*)mapped_host(sp, sizeof(double) * m * 3) : nullptr;
    if (mid && msp) {
        k_hist_in<<<blocks, 256, 0, st>>>(n, mid, msp, D.hid, D.hds);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        return SPHDEM_OK;
    }
    int r = ensure_xfer(H, m * 3 + (m + 1) / 2);
    if (r) return r;
    double* dsp = H->xfer;
    int* dids = (int*)(H->xfer + m * 3);
    if (set) {
        CK(cudaMemcpyAsync(dids, ids, sizeof(int) * m, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(dsp, sp, sizeof(double) * m * 3, cudaMemcpyHostToDevice, st));
        k_hist_in<<<blocks, 256, 0, st>>>(n, dids, dsp, D.hid, D.hds);
        CK(cudaGetLastError());
    } else {
        k_hist_out<<<blocks, 256, 0, st>>>(n, D.hid, D.hds, dids, dsp);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(ids, dids, sizeof(int) * m, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(sp, dsp, sizeof(double) * m * 3, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return SPHDEM_OK;
}

template <typename R>
static int mlp_state_t(SphdemHandle* H, float* params, double* stats, int32_t* trained, const float* pin,
                       const double* sin, int32_t tin, bool set) {
    EngineHost<R>* EH = (EngineHost<R>*)H->eng;
    if (!EH->has_mlp) return SPHDEM_E_ARG;
    CK(cudaStreamSynchronize(H->stream));
    if (set) {
        int r = mlp_put_params(EH->net, pin, H->stream);
        if (r) return r;
        CK(cudaMemcpy(EH->K.mstat, sin, sizeof(double) * MS_COUNT, cudaMemcpyHostToDevice));
        EH->mlp_trained = tin;
        CK(cudaStreamSynchronize(H->stream));
    } else {
        int r = mlp_get_params(EH->net, params);
        if (r) return r;
        CK(cudaMemcpy(stats, EH->K.mstat, sizeof(double) * MS_COUNT, cudaMemcpyDeviceToHost));
        *trained = EH->mlp_trained;
    }
    return SPHDEM_OK;
}

extern "C" int sphdem_get_mlp_state(SphdemHandle* h, float* params, double* stats, int32_t* trained_steps) {
    if (h && h->kind == 1) return SPHDEM_E_UNSUPPORTED;   // ISPH-DEM engine only
    if (!h || !h->committed || !params || !stats || !trained_steps) return SPHDEM_E_ARG;
    return h->prec == SPHDEM_PREC_FP64
               ? mlp_state_t<double>(h, params, stats, trained_steps, nullptr, nullptr, 0, false)
               : mlp_state_t<float>(h, params, stats, trained_steps, nullptr, nullptr, 0, false);
}

extern "C" int sphdem_set_mlp_state(SphdemHandle* h, const float* params, const double* stats,
                                    int32_t trained_steps) {
    if (h && h->kind == 1) return SPHDEM_E_UNSUPPORTED;   // ISPH-DEM engine only
    if (!h || !h->committed || !params || !stats || trained_steps < 0) return SPHDEM_E_ARG;
    return h->prec == SPHDEM_PREC_FP64
               ? mlp_state_t<double>(h, nullptr, nullptr, nullptr, params, stats, trained_steps, true)
               : mlp_state_t<float>(h, nullptr, nullptr, nullptr, params, stats, trained_steps, true);
}

extern "C" int sphdem_get_history(SphdemHandle* h, int32_t* ids, double* springs) {
    if (h && h->kind == 1) return SPHDEM_E_UNSUPPORTED;   // ISPH-DEM engine only
    if (!h || !ids || !springs || !h->committed) return SPHDEM_E_ARG;
    return h->prec == SPHDEM_PREC_FP64 ? history_t<double>(h, ids, springs, false)
                                       : history_t<float>(h, ids, springs, false);
}

extern "C" int sphdem_set_history(SphdemHandle* h, const int32_t* ids, const double* springs) {
    if (h && h->kind == 1) return SPHDEM_E_UNSUPPORTED;   // ISPH-DEM engine only
    if (!h || !ids || !springs || !h->committed) return SPHDEM_E_ARG;
    return h->prec == SPHDEM_PREC_FP64 ? history_t<double>(h, (int32_t*)ids, (double*)springs, true)
                                       : history_t<float>(h, (int32_t*)ids, (double*)springs, true);
}

extern "C" int sphdem_set_graphs(SphdemHandle* h, int on) {
    if (!h) return SPHDEM_E_ARG;
    CK(cudaStreamSynchronize(h->stream));
    h->use_graphs = on ? 1 : 0;
    return SPHDEM_OK;
}

extern "C" int sphdem_set_timing(SphdemHandle* h, int on) {
    if (!h) return SPHDEM_E_ARG;
    if (h->ev_beg.empty()) {
        h->ev_beg.resize(KT_COUNT);
        h->ev_end.resize(KT_COUNT);
        for (int k = 0; k < KT_COUNT; k++) {
            CK(cudaEventCreate(&h->ev_beg[k]));
            CK(cudaEventCreate(&h->ev_end[k]));
        }
        h->ev_used.assign(KT_COUNT, 0);
        h->kern_ms.assign(KT_COUNT, 0.0);
        h->kern_n.assign(KT_COUNT, 0);
    }
    if ((on != 0) != (h->timing != 0)) {
        // captured graphs embed (or omit) the event records: recapture
        CK(cudaStreamSynchronize(h->stream));
        for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
        h->graphs.clear();
        h->graph_launches.clear();
        h->graph_kused.clear();
    }
    h->timing = on ? 1 : 0;
    return SPHDEM_OK;
}

extern "C" int sphdem_set_timing_only(SphdemHandle* h, int k) {
    if (!h || k < -1 || k >= KT_COUNT) return SPHDEM_E_ARG;
    if (k != h->time_only) {
        CK(cudaStreamSynchronize(h->stream));
        for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
        h->graphs.clear();
        h->graph_launches.clear();
        h->graph_kused.clear();
    }
    h->time_only = k;
    return SPHDEM_OK;
}

extern "C" int sphdem_set_concurrency(SphdemHandle* h, int on) {
    if (!h) return SPHDEM_E_ARG;
    if ((on != 0) != (h->concurrent != 0)) {
        // the step graphs embed the fork (or not): recapture
        CK(cudaStreamSynchronize(h->stream));
        for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
        h->graphs.clear();
        h->graph_launches.clear();
        h->graph_kused.clear();
    }
    h->concurrent = on ? 1 : 0;
    return SPHDEM_OK;
}

extern "C" int sphdem_collect_timing(SphdemHandle* h) {
    if (!h || h->ev_beg.empty()) return SPHDEM_E_ARG;
    CK(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < KT_COUNT; k++) {
        if (!h->ev_used[k]) continue;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, h->ev_beg[k], h->ev_end[k]) == cudaSuccess) {
            h->kern_ms[k] += ms;
            h->kern_n[k] += 1;
        }
        h->ev_used[k] = 0;
    }
    return SPHDEM_OK;
}

extern "C" int sphdem_get_timing(SphdemHandle* h, int k, char* name, int name_cap, double* total_ms, int64_t* launches) {
    if (!h || k < 0) return SPHDEM_E_ARG;
    if (k >= KT_COUNT) return SPHDEM_E_ARG;
    if (name && name_cap > 0) {
        std::strncpy(name, KT_NAMES[k], name_cap - 1);
        name[name_cap - 1] = 0;
    }
    if (total_ms) *total_ms = h->kern_ms.empty() ? 0.0 : h->kern_ms[k];
    if (launches) *launches = h->kern_n.empty() ? 0 : h->kern_n[k];
    return SPHDEM_OK;
}

extern "C" int sphdem_write_vtk_dem(SphdemHandle* h, const char* path) {
    if (h && h->kind == 1) return SPHDEM_E_UNSUPPORTED;   // ISPH-DEM engine only
    if (!h || !path || !h->committed) return SPHDEM_E_ARG;
    int n = h->nd;
    std::vector<double> x(n), y(n), z(n), magf(n), eliz(n, 1.0), por(n), uz(n), qsd(n), ftz(n), temp(n), rad(n), dtemp(n);
    std::vector<int> itype(n), ptype(n), idx(n);
    int r = 0;
    size_t bd = sizeof(double) * n, bi = sizeof(int) * n;
    r |= sphdem_get_field(h, 1, SPHDEM_F_X, x.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_Y, y.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_Z, z.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_DEMPOR, por.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_UZ, uz.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_Q_SD, qsd.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_FTOTALZ, ftz.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_TEMP, temp.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_RAD, rad.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_DTEMP, dtemp.data(), bd);
    r |= sphdem_get_field(h, 1, SPHDEM_F_ITYPE, itype.data(), bi);
    r |= sphdem_get_field(h, 1, SPHDEM_F_PTYPE, ptype.data(), bi);
    r |= sphdem_get_field(h, 1, SPHDEM_F_DEM_IDX, idx.data(), bi);
    if (r) return SPHDEM_E_CUDA;
    if (n > 0) {
        if (h->prec == SPHDEM_PREC_FP64) {
            auto* EH = (EngineHost<double>*)h->eng;
            if (download_real<double>(magf.data(), EH->E.dw.magf, n, h->stream)) return SPHDEM_E_CUDA;
        } else {
            auto* EH = (EngineHost<float>*)h->eng;
            if (download_real<double>(magf.data(), EH->E.dw.magf, n, h->stream)) return SPHDEM_E_CUDA;
        }
    }
    return sphdem_io_write_vtk_dem(path, n, x.data(), y.data(), z.data(), itype.data(), ptype.data(), idx.data(),
                                   magf.data(), eliz.data(), por.data(), uz.data(), qsd.data(), ftz.data(),
                                   temp.data(), rad.data(), dtemp.data());
}

extern "C" int sphdem_write_vtk_fluid(SphdemHandle* h, const char* path) {
    if (h && h->kind == 1) return SPHDEM_E_UNSUPPORTED;   // ISPH-DEM engine only
    if (!h || !path || !h->committed) return SPHDEM_E_ARG;
    int n = h->ns;
    std::vector<double> x(n), y(n), z(n), por(n), pres(n), dtemp(n), rho(n), temp(n), uz(n);
    std::vector<int> ptype(n), btype(n);
    size_t bd = sizeof(double) * n, bi = sizeof(int) * n;
    int r = 0;
    r |= sphdem_get_field(h, 0, SPHDEM_F_X, x.data(), bd);
    r |= sphdem_get_field(h, 0, SPHDEM_F_Y, y.data(), bd);
    r |= sphdem_get_field(h, 0, SPHDEM_F_Z, z.data(), bd);
    r |= sphdem_get_field(h, 0, SPHDEM_F_DEMPOR, por.data(), bd);
    r |= sphdem_get_field(h, 0, SPHDEM_F_PRES, pres.data(), bd);
    r |= sphdem_get_field(h, 0, SPHDEM_F_DTEMP, dtemp.data(), bd);
    r |= sphdem_get_field(h, 0, SPHDEM_F_RHO, rho.data(), bd);
    r |= sphdem_get_field(h, 0, SPHDEM_F_TEMP, temp.data(), bd);
    r |= sphdem_get_field(h, 0, SPHDEM_F_UZ, uz.data(), bd);
    r |= sphdem_get_field(h, 0, SPHDEM_F_PTYPE, ptype.data(), bi);
    r |= sphdem_get_field(h, 0, SPHDEM_F_BUFFER_TYPE, btype.data(), bi);
    if (r) return SPHDEM_E_CUDA;
    return sphdem_io_write_vtk_fluid(path, n, ptype.data(), x.data(), y.data(), z.data(), por.data(), pres.data(),
                                     dtemp.data(), btype.data(), rho.data(), temp.data(), uz.data());
}

// ---------------------------------------------------------------------------
// asynchronous output: sphdem_snapshot / sphdem_write_snapshot
// ---------------------------------------------------------------------------
static const int SNAP_DEM[] = {SPHDEM_F_X, SPHDEM_F_Y, SPHDEM_F_Z, SPHDEM_F_DEMPOR, SPHDEM_F_UZ, SPHDEM_F_Q_SD,
                               SPHDEM_F_FTOTALZ, SPHDEM_F_TEMP, SPHDEM_F_RAD, SPHDEM_F_DTEMP, SPHDEM_F_ITYPE,
                               SPHDEM_F_PTYPE, SPHDEM_F_DEM_IDX};
static const int SNAP_SPH[] = {SPHDEM_F_X, SPHDEM_F_Y, SPHDEM_F_Z, SPHDEM_F_DEMPOR, SPHDEM_F_PRES, SPHDEM_F_DTEMP,
                               SPHDEM_F_RHO, SPHDEM_F_TEMP, SPHDEM_F_UZ, SPHDEM_F_PTYPE, SPHDEM_F_BUFFER_TYPE};
static const int SNAP_MAGF = -1;   // the DEM drag slip magnitude (no ABI field), packed after the fields

template <typename R>
static int snapshot_t(SphdemHandle* H) {
    auto* EH = (EngineHost<R>*)H->eng;
    cudaStream_t st = H->stream;
    if (!H->snap_stream) {
        CK(cudaStreamCreateWithFlags(&H->snap_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&H->snap_packed, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&H->snap_done, cudaEventDisableTiming));
    }
    // the previous snapshot's copy must be out of the buffers first
    if (H->snap_pending) CK(cudaEventSynchronize(H->snap_done));
    std::vector<SphdemHandle::SnapField> fl;
    std::vector<const void*> src;
    size_t off = 0;
    auto add = [&](int which, int field, const void* ptr, int kind, int n) {
        size_t es = kind == 0 ? sizeof(double) : kind == 1 ? sizeof(R) : sizeof(int);
        size_t b = es * (size_t)n;
        fl.push_back({which, field, kind, off, b});
        src.push_back(ptr);
        off += (b + 255) & ~(size_t)255;
    };
    for (int w = 0; w < 2; w++) {
        const int* list = w ? SNAP_DEM : SNAP_SPH;
        int cnt = w ? (int)(sizeof(SNAP_DEM) / sizeof(int)) : (int)(sizeof(SNAP_SPH) / sizeof(int));
        int n = w ? H->nd : H->ns;
        for (int k = 0; k < cnt; k++) {
            const void* ptr;
            int kind;
            if (field_ptr<R>(H, w, list[k], &ptr, &kind)) return SPHDEM_E_ARG;
            add(w, list[k], ptr, kind, n);
        }
    }
    add(1, SNAP_MAGF, EH->E.dw.magf, 0, H->nd);
    if (off > H->snap_bytes) {
        if (H->snap_dev) CK(cudaFree(H->snap_dev));
        if (H->snap_host) CK(cudaFreeHost(H->snap_host));
        H->snap_dev = nullptr;
        H->snap_host = nullptr;
        H->snap_bytes = 0;
        if (cudaMalloc(&H->snap_dev, off) != cudaSuccess) return SPHDEM_E_NOMEM;
        if (cudaMallocHost(&H->snap_host, off) != cudaSuccess) return SPHDEM_E_NOMEM;
        H->snap_bytes = off;
    }
    // pack on the step stream: ordered after the steps so far, before the next
    for (size_t k = 0; k < fl.size(); k++)
        if (fl[k].bytes)
            CK(cudaMemcpyAsync(H->snap_dev + fl[k].off, src[k], fl[k].bytes, cudaMemcpyDeviceToDevice, st));
    CK(cudaEventRecord(H->snap_packed, st));
    // copy out on the output stream while the next steps run
    CK(cudaStreamWaitEvent(H->snap_stream, H->snap_packed, 0));
    CK(cudaMemcpyAsync(H->snap_host, H->snap_dev, off, cudaMemcpyDeviceToHost, H->snap_stream));
    CK(cudaEventRecord(H->snap_done, H->snap_stream));
    H->snap_fields = fl;
    H->snap_pending = true;
    H->snap_t_ref = EH->E.P.t_ref;
    H->snap_count = H->count;
    H->snap_time = H->time;
    return SPHDEM_OK;
}

extern "C" int sphdem_snapshot(SphdemHandle* h) {
    if (h && h->kind == 1) return SPHDEM_E_UNSUPPORTED;   // ISPH-DEM engine only
    if (!h || !h->committed) return SPHDEM_E_ARG;
    return h->prec == SPHDEM_PREC_FP64 ? snapshot_t<double>(h) : snapshot_t<float>(h);
}

extern "C" int sphdem_write_snapshot(SphdemHandle* h, const char* dem_vtk_path, const char* fluid_vtk_path) {
    if (!h || !h->snap_pending) return SPHDEM_E_ARG;
    CK(cudaEventSynchronize(h->snap_done));
    const bool f32 = h->prec != SPHDEM_PREC_FP64;
    auto real = [&](int which, int field, double off) {
        std::vector<double> v;
        for (auto& f : h->snap_fields) {
            if (f.which != which || f.field != field) continue;
            const unsigned char* p = h->snap_host + f.off;
            size_t es = f.kind == 0 ? 8 : (f.kind == 1 ? (f32 ? 4 : 8) : 4);
            size_t n = f.bytes / es;
            v.resize(n);
            for (size_t i = 0; i < n; i++) {
                if (f.kind == 0 || (f.kind == 1 && !f32)) v[i] = ((const double*)p)[i] + off;
                else v[i] = (double)((const float*)p)[i] + off;
            }
        }
        return v;
    };
    auto ints = [&](int which, int field) {
        std::vector<int> v;
        for (auto& f : h->snap_fields)
            if (f.which == which && f.field == field) {
                v.resize(f.bytes / 4);
                std::memcpy(v.data(), h->snap_host + f.off, f.bytes);
            }
        return v;
    };
    int r = SPHDEM_OK;
    if (dem_vtk_path) {
        int n = h->nd;
        auto x = real(1, SPHDEM_F_X, 0), y = real(1, SPHDEM_F_Y, 0), z = real(1, SPHDEM_F_Z, 0);
        auto por = real(1, SPHDEM_F_DEMPOR, 0), uz = real(1, SPHDEM_F_UZ, 0), qsd = real(1, SPHDEM_F_Q_SD, 0);
        auto ftz = real(1, SPHDEM_F_FTOTALZ, 0), temp = real(1, SPHDEM_F_TEMP, 0), rad = real(1, SPHDEM_F_RAD, 0);
        auto dtemp = real(1, SPHDEM_F_DTEMP, 0), magf = real(1, SNAP_MAGF, 0);
        auto it = ints(1, SPHDEM_F_ITYPE), pt = ints(1, SPHDEM_F_PTYPE), idx = ints(1, SPHDEM_F_DEM_IDX);
        std::vector<double> eliz(n, 1.0);
        r = sphdem_io_write_vtk_dem(dem_vtk_path, n, x.data(), y.data(), z.data(), it.data(), pt.data(), idx.data(),
                                    magf.data(), eliz.data(), por.data(), uz.data(), qsd.data(), ftz.data(),
                                    temp.data(), rad.data(), dtemp.data());
        if (r) return r;
    }
    if (fluid_vtk_path) {
        int n = h->ns;
        auto x = real(0, SPHDEM_F_X, 0), y = real(0, SPHDEM_F_Y, 0), z = real(0, SPHDEM_F_Z, 0);
        auto por = real(0, SPHDEM_F_DEMPOR, 0), pres = real(0, SPHDEM_F_PRES, 0), dtemp = real(0, SPHDEM_F_DTEMP, 0);
        auto rho = real(0, SPHDEM_F_RHO, 0), temp = real(0, SPHDEM_F_TEMP, h->snap_t_ref), uz = real(0, SPHDEM_F_UZ, 0);
        auto pt = ints(0, SPHDEM_F_PTYPE), bt = ints(0, SPHDEM_F_BUFFER_TYPE);
        r = sphdem_io_write_vtk_fluid(fluid_vtk_path, n, pt.data(), x.data(), y.data(), z.data(), por.data(),
                                      pres.data(), dtemp.data(), bt.data(), rho.data(), temp.data(), uz.data());
    }
    return r;
}

extern "C" int sphdem_write_restart(SphdemHandle* h, const char* path) {
    if (h && h->kind == 1) return SPHDEM_E_UNSUPPORTED;   // ISPH-DEM engine only
    if (!h || !path || !h->committed) return SPHDEM_E_ARG;
    FILE* f = std::fopen(path, "w");
    if (!f) return SPHDEM_E_INPUT;
    // every column the reader understands, tab-separated labels
    const int lbl[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35};
    const int fld[] = {SPHDEM_F_X, SPHDEM_F_Y, SPHDEM_F_Z, SPHDEM_F_UX, SPHDEM_F_UY, SPHDEM_F_UZ, SPHDEM_F_M,
                       SPHDEM_F_PTYPE, SPHDEM_F_H, SPHDEM_F_TEMP, SPHDEM_F_PRES, SPHDEM_F_RHO, SPHDEM_F_FLT_S,
                       SPHDEM_F_RAD, SPHDEM_F_RI, SPHDEM_F_DEM_IDX, SPHDEM_F_WX, SPHDEM_F_WY, SPHDEM_F_WZ,
                       SPHDEM_F_TEMP1, SPHDEM_F_TEMP2, SPHDEM_F_TEMP3};
    const int nc = sizeof(lbl) / sizeof(lbl[0]);
    for (int c = 0; c < nc; c++) std::fprintf(f, c ? "\t%d" : "%d", lbl[c]);
    std::fprintf(f, "\n");
    for (int q = 0; q < 2; q++) {
        int n = q ? h->nd : h->ns;
        if (n == 0) continue;
        std::vector<std::vector<double>> cols(nc, std::vector<double>(n, 0.0));
        for (int c = 0; c < nc; c++) {
            int fd = fld[c];
            if (is_int_field(fd)) {
                if (q == 0 && fd == SPHDEM_F_DEM_IDX) continue;
                std::vector<int> v(n);
                if (sphdem_get_field(h, q, fd, v.data(), sizeof(int) * n) == 0)
                    for (int i = 0; i < n; i++) cols[c][i] = v[i];
            } else {
                std::vector<double> v(n);
                if (sphdem_get_field(h, q, fd, v.data(), sizeof(double) * n) == 0) cols[c] = v;
            }
        }
        for (int i = 0; i < n; i++) {
            for (int c = 0; c < nc; c++) {
                if (fld[c] == SPHDEM_F_PTYPE || fld[c] == SPHDEM_F_DEM_IDX)
                    std::fprintf(f, c ? "\t%d" : "%d", (int)cols[c][i]);
                else
                    std::fprintf(f, c ? "\t%.17g" : "%.17g", cols[c][i]);
            }
            std::fprintf(f, "\n");
        }
    }
    std::fclose(f);
    return SPHDEM_OK;
}

extern "C" int sphdem_get_time(SphdemHandle* h, double* time, int32_t* count) {
    if (!h || !time || !count) return SPHDEM_E_ARG;
    *time = h->time;
    *count = h->count;
    return SPHDEM_OK;
}

// ---------------------------------------------------------------------------
// slab exchange of a spatially sharded bed (slab.cuh)
// ---------------------------------------------------------------------------
extern "C" int sphdem_set_list_build(SphdemHandle* h, int32_t mode) {
    if (!h || h->committed || h->kind != 0) return SPHDEM_E_ARG;
    if (mode != 0 && mode != 1 && mode != 2 && mode != 4 && mode != 8) return SPHDEM_E_ARG;
    h->list_build_req = mode;
    return SPHDEM_OK;
}

extern "C" int sphdem_get_list_build(SphdemHandle* h, int32_t* mode) {
    if (!h || !mode || !h->committed || h->kind != 0) return SPHDEM_E_ARG;
    *mode = h->prec == SPHDEM_PREC_FP64 ? ((EngineHost<double>*)h->eng)->list_mode
                                        : ((EngineHost<float>*)h->eng)->list_mode;
    return SPHDEM_OK;
}

extern "C" int sphdem_set_beds(SphdemHandle* h, int32_t nbeds, const SphdemBedRow* rows) {
    if (!h || !rows || h->committed || h->kind != 0) return SPHDEM_E_ARG;
    if (h->p.dim != 2 || h->p.solver_type != SPHDEM_ISPH) return SPHDEM_E_UNSUPPORTED;
    if (nbeds < 1 || nbeds > SPHDEM_MAX_BEDS) return SPHDEM_E_ARG;
    std::vector<SphdemBedRow> b(rows, rows + nbeds);
    for (const SphdemBedRow& r : b) {
        const double v[7] = {r.y, r.inlet_uz, r.inlet_temp, r.obc_L1, r.obc_L2, r.obc_L3, r.obc_L4};
        for (double x : v)
            if (!std::isfinite(x)) return SPHDEM_E_ARG;
    }
    std::stable_sort(b.begin(), b.end(), [](const SphdemBedRow& a, const SphdemBedRow& c) { return a.y < c.y; });
    h->beds = b;
    return SPHDEM_OK;
}

extern "C" int sphdem_set_domain(SphdemHandle* h, const double* bbox6, double h0, double t_ref) {
    if (!h || !bbox6 || h->committed || h->kind != 0) return SPHDEM_E_ARG;
    if (!(h0 > 0) || !std::isfinite(t_ref)) return SPHDEM_E_ARG;
    for (int k = 0; k < 3; k++)
        if (!(bbox6[2 * k + 1] >= bbox6[2 * k])) return SPHDEM_E_ARG;
    for (int k = 0; k < 6; k++) h->dom_bbox[k] = bbox6[k];
    h->dom_h0 = h0;
    h->dom_tref = (double)(float)t_ref;
    h->dom_set = true;
    return SPHDEM_OK;
}

extern "C" int sphdem_bed_domain(const SphdemParams* p, const double* sx, const double* sy, const double* sz,
                                  const double* sh, const double* stemp, int32_t ns, const double* dx,
                                  const double* dy, const double* dz, const double* dh, int32_t nd, double* bbox6,
                                  double* h0, double* t_ref) {
    if (!p || !bbox6 || !h0 || !t_ref || ns < 0 || nd < 0 || ns + nd == 0) return SPHDEM_E_ARG;
    if ((ns > 0 && (!sx || !sy || !sz || !sh || !stemp)) || (nd > 0 && (!dx || !dy || !dz || !dh))) return SPHDEM_E_ARG;
    std::vector<double> fx(sx, sx + ns), fy(sy, sy + ns), fz(sz, sz + ns);
    fx.insert(fx.end(), dx, dx + nd);
    fy.insert(fy.end(), dy, dy + nd);
    fz.insert(fz.end(), dz, dz + nd);
    bed_box(*p, fx.data(), fy.data(), fz.data(), ns + nd, bbox6);
    *h0 = ns > 0 ? sh[0] : dh[0];
    double s = 0;
    for (int i = 0; i < ns; i++) s += stemp[i];
    *t_ref = ns > 0 ? (double)(float)(s / (double)ns) : 0.0;
    if (!std::isfinite(*t_ref)) *t_ref = 0.0;
    return SPHDEM_OK;
}

extern "C" int sphdem_slab_record_bytes(int which) {
    return which == SPHDEM_SPH ? SLAB_SPH_BYTES : (which == SPHDEM_DEM ? SLAB_DEM_BYTES : SPHDEM_E_ARG);
}

namespace {

template <typename R>
SphCur<R> sph_cur(SphdemHandle* H) {
    EngineHost<R>* EH = (EngineHost<R>*)H->eng;
    Engine<R>& E = EH->E;
    SphState<R>& S = E.S[E.cur_s];
    SphWork<R>& W = E.sw;
    const bool xs = E.P.xsph;
    SphCur<R> C;
    C.x = S.x; C.y = S.y; C.z = S.z; C.h = S.h;
    C.ux = xs ? W.u_tmpx : S.ux; C.uy = xs ? W.u_tmpy : S.uy; C.uz = xs ? W.u_tmpz : S.uz;
    C.temp = xs ? W.temp_tmp : S.temp;
    C.m = W.m_new; C.rho = W.rho_new; C.pres = W.p_new;
    C.dDEMpor = S.dDEMpor; C.flt_s = S.flt_s;
    C.ptype = S.ptype; C.btype = S.btype; C.itype = S.itype; C.pid = S.pid;
    C.t_ref = E.P.t_ref;
    return C;
}

// positions and i_type of the current state of one set
template <typename R>
void set_xyzi(SphdemHandle* H, int which, const double** x, const double** y, const double** z, int** it, int* n) {
    EngineHost<R>* EH = (EngineHost<R>*)H->eng;
    Engine<R>& E = EH->E;
    if (which == SPHDEM_SPH) {
        SphState<R>& S = E.S[E.cur_s];
        *x = S.x; *y = S.y; *z = S.z; *it = S.itype; *n = E.P.ns;
    } else {
        DemState<double>& D = E.D[E.cur_d];
        *x = D.x; *y = D.y; *z = D.z; *it = D.itype; *n = E.P.nd;
    }
}

const DevParams& dev_params(SphdemHandle* H) {
    return H->prec == SPHDEM_PREC_FP64 ? ((EngineHost<double>*)H->eng)->E.P : ((EngineHost<float>*)H->eng)->E.P;
}

// slots of one set selected by mode (0: active with layer in [lo, hi); 1:
// parked), ascending, into slots[0, cap); the count to *count (host)
int slab_select(SphdemHandle* H, int which, int axis, int lo, int hi, int mode, int* slots, int cap, int* count) {
    const double *x, *y, *z;
    int* it;
    int n;
    if (H->prec == SPHDEM_PREC_FP64) set_xyzi<double>(H, which, &x, &y, &z, &it, &n);
    else set_xyzi<float>(H, which, &x, &y, &z, &it, &n);
    const DevParams& P = dev_params(H);
    cudaStream_t st = H->stream;
    int nb = std::max(1, nblocks(n, TPB));
    if (nb > H->slab_blk_n) {
        if (H->slab_blk) CK(cudaFree(H->slab_blk));
        CK(cudaMalloc(&H->slab_blk, sizeof(int) * nb));
        H->slab_blk_n = nb;
    }
    if (!H->slab_tot) CK(cudaMalloc(&H->slab_tot, sizeof(int)));
    k_slab_flag<<<nb, TPB, 0, st>>>(P, n, x, y, z, it, axis, lo, hi, mode, H->slab_blk);
    k_slab_scan<<<1, 1024, 0, st>>>(nb, H->slab_blk, H->slab_tot);
    k_slab_compact<<<nb, TPB, 0, st>>>(P, n, x, y, z, it, axis, lo, hi, mode, H->slab_blk, slots, cap);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(count, H->slab_tot, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SPHDEM_OK;
}

}  // namespace

extern "C" int sphdem_slab_select(SphdemHandle* h, int which, int axis, int32_t lo, int32_t hi, int32_t* d_slots,
                                  int32_t cap, int32_t* count) {
    if (!h || !h->committed || h->kind != 0 || !count || axis < 0 || axis > 2) return SPHDEM_E_ARG;
    if (which != SPHDEM_SPH && which != SPHDEM_DEM) return SPHDEM_E_ARG;
    if (cap > 0 && !d_slots) return SPHDEM_E_ARG;
    return slab_select(h, which, axis, lo, hi, 0, d_slots, cap, count);
}

extern "C" int sphdem_slab_export(SphdemHandle* h, int which, const int32_t* d_slots, int32_t n, void* d_buf) {
    if (!h || !h->committed || h->kind != 0 || n < 0 || (n > 0 && (!d_slots || !d_buf))) return SPHDEM_E_ARG;
    if (n == 0) return SPHDEM_OK;
    cudaStream_t st = h->stream;
    unsigned char* buf = (unsigned char*)d_buf;
    if (which == SPHDEM_SPH) {
        if (h->prec == SPHDEM_PREC_FP64) k_slab_export_sph<double><<<nblocks(n, TPB), TPB, 0, st>>>(sph_cur<double>(h), d_slots, n, buf);
        else k_slab_export_sph<float><<<nblocks(n, TPB), TPB, 0, st>>>(sph_cur<float>(h), d_slots, n, buf);
    } else if (which == SPHDEM_DEM) {
        if (h->prec == SPHDEM_PREC_FP64) {
            Engine<double>& E = ((EngineHost<double>*)h->eng)->E;
            k_slab_export_dem<<<nblocks(n, TPB), TPB, 0, st>>>(E.D[E.cur_d], E.P.nd, d_slots, n, buf);
        } else {
            Engine<float>& E = ((EngineHost<float>*)h->eng)->E;
            k_slab_export_dem<<<nblocks(n, TPB), TPB, 0, st>>>(E.D[E.cur_d], E.P.nd, d_slots, n, buf);
        }
    } else {
        return SPHDEM_E_ARG;
    }
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

extern "C" int sphdem_slab_keep(SphdemHandle* h, int which, int axis, int32_t lo, int32_t hi) {
    if (!h || !h->committed || h->kind != 0 || axis < 0 || axis > 2) return SPHDEM_E_ARG;
    if (which != SPHDEM_SPH && which != SPHDEM_DEM) return SPHDEM_E_ARG;
    const double *x, *y, *z;
    int* it;
    int n;
    if (h->prec == SPHDEM_PREC_FP64) set_xyzi<double>(h, which, &x, &y, &z, &it, &n);
    else set_xyzi<float>(h, which, &x, &y, &z, &it, &n);
    if (n == 0) return SPHDEM_OK;
    k_slab_keep<<<nblocks(n, TPB), TPB, 0, h->stream>>>(dev_params(h), n, x, y, z, it, axis, lo, hi);
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

extern "C" int sphdem_slab_import(SphdemHandle* h, int which, const void* d_buf, int32_t n) {
    if (!h || !h->committed || h->kind != 0 || n < 0 || (n > 0 && !d_buf)) return SPHDEM_E_ARG;
    if (which != SPHDEM_SPH && which != SPHDEM_DEM) return SPHDEM_E_ARG;
    if (n == 0) return SPHDEM_OK;
    if (n > h->slab_free_n) {
        if (h->slab_free) CK(cudaFree(h->slab_free));
        CK(cudaMalloc(&h->slab_free, sizeof(int) * n));
        h->slab_free_n = n;
    }
    // the first n parked slots, ascending
    int parked = 0;
    int r = slab_select(h, which, 0, 0, 0, 1, h->slab_free, n, &parked);
    if (r) return r;
    if (parked < n) return SPHDEM_E_NOMEM;
    cudaStream_t st = h->stream;
    const unsigned char* buf = (const unsigned char*)d_buf;
    if (which == SPHDEM_SPH) {
        if (h->prec == SPHDEM_PREC_FP64) k_slab_import_sph<double><<<nblocks(n, TPB), TPB, 0, st>>>(sph_cur<double>(h), h->slab_free, n, buf);
        else k_slab_import_sph<float><<<nblocks(n, TPB), TPB, 0, st>>>(sph_cur<float>(h), h->slab_free, n, buf);
    } else {
        if (h->prec == SPHDEM_PREC_FP64) {
            Engine<double>& E = ((EngineHost<double>*)h->eng)->E;
            k_slab_import_dem<<<nblocks(n, TPB), TPB, 0, st>>>(E.D[E.cur_d], E.P.nd, h->slab_free, n, buf);
        } else {
            Engine<float>& E = ((EngineHost<float>*)h->eng)->E;
            k_slab_import_dem<<<nblocks(n, TPB), TPB, 0, st>>>(E.D[E.cur_d], E.P.nd, h->slab_free, n, buf);
        }
    }
    CK(cudaGetLastError());
    return SPHDEM_OK;
}

extern "C" int sphdem_slab_active(SphdemHandle* h, int which, int32_t* n_active) {
    if (!h || !h->committed || h->kind != 0 || !n_active) return SPHDEM_E_ARG;
    if (which != SPHDEM_SPH && which != SPHDEM_DEM) return SPHDEM_E_ARG;
    int parked = 0;
    int r = slab_select(h, which, 0, 0, 0, 1, nullptr, 0, &parked);
    if (r) return r;
    *n_active = (which == SPHDEM_SPH ? h->ns : h->nd) - parked;
    return SPHDEM_OK;
}

extern "C" int sphdem_get_counts(SphdemHandle* h, int32_t* ns, int32_t* nd) {
    if (!h || !ns || !nd) return SPHDEM_E_ARG;
    *ns = h->ns;
    *nd = h->nd;
    return SPHDEM_OK;
}

extern "C" int sphdem_get_stream(SphdemHandle* h, void** stream) {
    if (!h || !stream) return SPHDEM_E_ARG;
    *stream = (void*)h->stream;
    return SPHDEM_OK;
}

extern "C" int sphdem_get_launch_count(SphdemHandle* h, int64_t* launches) {
    if (!h || !launches) return SPHDEM_E_ARG;
    *launches = h->last_launches;
    return SPHDEM_OK;
}

extern "C" void sphdem_destroy(SphdemHandle* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
    for (cudaEvent_t e : h->ev_beg) cudaEventDestroy(e);
    for (cudaEvent_t e : h->ev_end) cudaEventDestroy(e);
    if (h->eng) engine_destroy(h);
    if (h->xfer) cudaFree(h->xfer);
    if (h->snap_stream) cudaStreamSynchronize(h->snap_stream);
    if (h->snap_dev) cudaFree(h->snap_dev);
    if (h->snap_host) cudaFreeHost(h->snap_host);
    if (h->snap_packed) cudaEventDestroy(h->snap_packed);
    if (h->snap_done) cudaEventDestroy(h->snap_done);
    if (h->snap_stream) cudaStreamDestroy(h->snap_stream);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->slab_blk) cudaFree(h->slab_blk);
    if (h->slab_tot) cudaFree(h->slab_tot);
    if (h->slab_free) cudaFree(h->slab_free);
    if (h->d_beds) cudaFree(h->d_beds);
    if (h->dem_stream) cudaStreamDestroy(h->dem_stream);
    for (cudaEvent_t e : h->fork_ev)
        if (e) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

extern "C" const char* sphdem_strerror(int s) {
    switch (s) {
    case SPHDEM_OK: return "ok";
    case SPHDEM_E_ARG: return "invalid argument";
    case SPHDEM_E_CUDA: return "CUDA runtime error";
    case SPHDEM_E_INPUT: return "malformed input";
    case SPHDEM_E_OVERFLOW: return "neighbour list or contact history overflow";
    case SPHDEM_E_NAN: return "non-finite value in the particle state";
    case SPHDEM_E_TIMEOUT: return "bounded device wait timed out";
    case SPHDEM_E_UNSUPPORTED: return "switch combination not supported";
    case SPHDEM_E_NOMEM: return "out of memory or size above limit";
    }
    return "unknown status";
}

extern "C" int sphdem_params_size(void) { return (int)sizeof(SphdemParams); }
