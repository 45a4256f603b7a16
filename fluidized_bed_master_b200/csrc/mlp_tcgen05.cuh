// mlp_tcgen05.cuh -- the per-particle MLP of the learned PPE warm start on
// the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Network: 16 -> 64 -> 64 -> 1, ReLU, BF16 weights and activations, FP32
// accumulation in tensor memory (TMEM).  A CTA of 128 threads owns one SM
// and walks tiles of 128 particles (the MMA's M):
//
//   X   [128 x 16]  --tcgen05.mma-->  D1 = X W1^T   (TMEM columns   0.. 63)
//   H1 = relu(D1 + b1) -> BF16 smem
//   H1  [128 x 64]  --tcgen05.mma-->  D2 = H1 W2^T  (TMEM columns  64..127)
//   y  = relu(D2 + b2) . w3 + b3      (per-thread dot on the CUDA cores)
//
// The gradient kernel adds, per tile,
//   delta2 = dL/dz2 = dL/dy w3 (z2 > 0)               -> BF16 smem
//   D3 = delta2 W2                                     (TMEM columns   0.. 63)
//   delta1 = D3 (z1 > 0)                               -> BF16 smem
//   [dW2 | db2] += delta2^T [H1 | 1]  (M = 128: 64 units + 64 zero rows,
//                  N = 80, K = the tile's 128 particles) (columns 128..207)
//   [dW1 | db1] += delta1^T [X | 1]   (N = 32)           (columns 208..239)
// (the appended row of ones turns the bias sums into MMA columns), and
// accumulates dw3, db3 and the loss in registers (warp shuffles at the end).
// Each CTA writes its partial gradient; k_mlp_adam adds the partials in
// CTA order (deterministic) and takes one Adam step on FP32 master weights.
//
// Operand layout in shared memory: the canonical no-swizzle K-major layout
// of the tcgen05 matrix descriptor.  A [R x K] BF16 operand is stored as
// 8-row x 16-byte core matrices, K-groups fastest:
//   byte(r, k) = ((r/8)(K/8) + k/8) 128 + (r%8) 16 + (k%8) 2
// so LBO (next core matrix along K) = 128 B and SBO (next 8-row group) =
// (K/8) 128 B; one MMA consumes K = 16 and the next K-slice starts 256 B on.
//
// Every mbarrier wait is bounded by the global timer; on a timeout the
// kernel records the failure in *err, stops issuing work, and frees its
// TMEM before returning.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sphdem {

constexpr int MLP_IN = 16, MLP_H = 64, MLP_TILE = 128;
// flattened FP32 parameter vector: W1 | b1 | W2 | b2 | w3 | b3
constexpr int MLP_OFF_W1 = 0, MLP_OFF_B1 = MLP_OFF_W1 + MLP_H * MLP_IN, MLP_OFF_W2 = MLP_OFF_B1 + MLP_H,
              MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H, MLP_OFF_W3 = MLP_OFF_B2 + MLP_H,
              MLP_OFF_B3 = MLP_OFF_W3 + MLP_H, MLP_NPARAM = MLP_OFF_B3 + 1;
constexpr int MLP_PART = MLP_NPARAM + 3;   // + loss, weight sum, pad
constexpr uint64_t MLP_WAIT_NS = 200000000ull;   // 0.2 s per wait

// device copies of the network the MMAs read
struct MlpDev {
    const __nv_bfloat16* W1;    // [64][16]  row n = hidden unit, K-major
    const __nv_bfloat16* W2;    // [64][64]  row n = layer-2 unit
    const __nv_bfloat16* W2T;   // [64][64]  W2 transposed (backward operand)
    const float* b1;
    const float* b2;
    const float* w3;            // BF16-rounded values held as float
    const float* b3;
};

// ---- PTX wrappers ---------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void tc_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tc_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] B[smem]^T, kind::f16 (BF16 in, FP32 accumulate)
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// bounded wait for the phase with the given parity; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity) {
    uint32_t addr = smem_u32(m);
    uint64_t t0 = global_ns();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, P;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > MLP_WAIT_NS) return false;
    }
}

// ---- descriptors ------------------------------------------------------------
__device__ __forceinline__ uint64_t smem_desc(const void* base, uint32_t lbo, uint32_t sbo) {
    uint32_t a = smem_u32(base);
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// kind::f16, BF16 A and B (K-major), FP32 D, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// byte offset of element (r, k) in an [R x K] core-matrix operand
__host__ __device__ __forceinline__ uint32_t cm_off(int r, int k, int K) {
    return (uint32_t)((((r >> 3) * (K >> 3) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// store 8 consecutive K-elements (16 B) of row r
__device__ __forceinline__ void st_row8(unsigned char* tile, int r, int k0, int K, const float* v) {
    __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]), p1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(v[4], v[5]), p3 = __floats2bfloat162_rn(v[6], v[7]);
    uint4 u;
    u.x = *reinterpret_cast<uint32_t*>(&p0);
    u.y = *reinterpret_cast<uint32_t*>(&p1);
    u.z = *reinterpret_cast<uint32_t*>(&p2);
    u.w = *reinterpret_cast<uint32_t*>(&p3);
    *reinterpret_cast<uint4*>(tile + cm_off(r, k0, K)) = u;
}
__device__ __forceinline__ void st_bf16(unsigned char* tile, int r, int k, int K, float v) {
    *reinterpret_cast<__nv_bfloat16*>(tile + cm_off(r, k, K)) = __float2bfloat16_rn(v);
}

// copy a row-major [R x K] BF16 matrix from global into core-matrix layout
__device__ __forceinline__ void load_operand(unsigned char* tile, const __nv_bfloat16* g, int R, int K) {
    for (int q = threadIdx.x; q < R * K / 8; q += blockDim.x) {
        int r = q / (K / 8), k0 = (q % (K / 8)) * 8;
        *reinterpret_cast<uint4*>(tile + cm_off(r, k0, K)) = *reinterpret_cast<const uint4*>(g + r * K + k0);
    }
}

// ---- shared-memory plan ------------------------------------------------------
// (offsets in bytes from a 1024-aligned base)
constexpr int SM_X = 0;                         // X   [128 x 16]       4 KB
constexpr int SM_W1 = SM_X + 4096;              // W1  [64 x 16]        2 KB
constexpr int SM_W2 = SM_W1 + 2048;             // W2  [64 x 64]        8 KB
constexpr int SM_H1 = SM_W2 + 8192;             // H1  [128 x 64]      16 KB
constexpr int SM_VEC = SM_H1 + 16384;           // b1, b2, w3 (FP32)   768 B
constexpr int SM_INFER_END = SM_VEC + 1024;     // inference total    ~31 KB
constexpr int SM_W2T = SM_INFER_END;            // W2T [64 x 64]        8 KB
constexpr int SM_XT = SM_W2T + 8192;            // [X^T; 1; 0] [32 x 128]   8 KB
constexpr int SM_H1T = SM_XT + 8192;            // [H1^T; 1; 0] [80 x 128] 20 KB
constexpr int SM_D2 = SM_H1T + 20480;           // delta2 [128 x 64]   16 KB
constexpr int SM_D2T = SM_D2 + 16384;           // delta2^T [128 x 128], rows 64.. zero  32 KB
constexpr int SM_D1T = SM_D2T + 32768;          // delta1^T [128 x 128], rows 64.. zero  32 KB
constexpr int SM_TRAIN_END = SM_D1T + 32768;    // training total     ~167 KB
constexpr int SM_ALIGN = 1024;
// TMEM columns of the gradient kernel
constexpr int TM_D1 = 0, TM_D2 = 64, TM_GW2 = 128, TM_GW1 = 208;
constexpr int GW2_N = 80, GW1_N = 32;   // dW2 | db2 | 0..,  dW1 | db1 | 0..

__device__ __forceinline__ unsigned char* smem_base(unsigned char* raw) {
    uintptr_t a = (uintptr_t)raw;
    uintptr_t s = (uintptr_t)__cvta_generic_to_shared(raw);
    uintptr_t pad = (SM_ALIGN - (s & (SM_ALIGN - 1))) & (SM_ALIGN - 1);
    return (unsigned char*)(a + pad);
}

__device__ __forceinline__ void load_vectors(float* v, const MlpDev& net) {
    for (int c = threadIdx.x; c < MLP_H; c += blockDim.x) {
        v[c] = net.b1[c];
        v[MLP_H + c] = net.b2[c];
        v[2 * MLP_H + c] = net.w3[c];
    }
}

// X tile row `tid` (zero past n); returns the row's features as float
__device__ __forceinline__ void load_x_row(unsigned char* sm, const __nv_bfloat16* feat, int n, int row, int tid,
                                           float* x) {
    if (row < n) {
        const uint4* src = reinterpret_cast<const uint4*>(feat + (size_t)row * MLP_IN);
        uint4 a = src[0], b = src[1];
        *reinterpret_cast<uint4*>(sm + SM_X + cm_off(tid, 0, MLP_IN)) = a;
        *reinterpret_cast<uint4*>(sm + SM_X + cm_off(tid, 8, MLP_IN)) = b;
        const __nv_bfloat16* pa = reinterpret_cast<const __nv_bfloat16*>(&a);
        const __nv_bfloat16* pb = reinterpret_cast<const __nv_bfloat16*>(&b);
#pragma unroll
        for (int q = 0; q < 8; q++) {
            x[q] = __bfloat162float(pa[q]);
            x[8 + q] = __bfloat162float(pb[q]);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 16; q++) x[q] = 0.f;
        st_row8(sm + SM_X, tid, 0, MLP_IN, x);
        st_row8(sm + SM_X, tid, 8, MLP_IN, x + 8);
    }
}

// one MMA group + commit by thread 0, bounded wait by all.  A thread whose
// wait runs out sets fail and remembers the phase (fparity: bit 1 = failed,
// bit 0 = parity), so that before freeing TMEM it can wait once more, again
// bounded, for an MMA group that may still be in flight.  stall (inference
// only; see k_mlp_infer) withholds the group and its commit, so nothing ever
// arrives on the barrier.
#define MLP_SYNC_ISSUE(...)                          \
    do {                                             \
        fence_async_smem();                          \
        tc_fence_before();                           \
        __syncthreads();                             \
        if (tid == 0 && !fail && !stall) {           \
            tc_fence_after();                        \
            __VA_ARGS__;                             \
            tc_commit(&mbar);                        \
        }                                            \
        __syncthreads();                             \
        if (!fail && !mbar_wait(&mbar, phase)) {     \
            fail = 1;                                \
            fparity = 2u | phase;                    \
        }                                            \
        phase ^= 1;                                  \
        tc_fence_after();                            \
    } while (0)

// the end of a kernel that may have given up on a wait: one more bounded wait
// for the group in flight, then every thread is past its last TMEM access
#define MLP_DRAIN()                                          \
    do {                                                     \
        if (fparity & 2u) mbar_wait(&mbar, fparity & 1u);    \
    } while (0)

// ---- inference --------------------------------------------------------------
// out[i] = MLP(feat[i]) for i < n; feat is row-major [n x 16] BF16.
// stall != 0 is the failure drill of the bounded waits: the first MMA group
// is not issued, its wait runs out after MLP_WAIT_NS, and the kernel must
// report through *err, free its TMEM and return (no MMA is in flight).
__global__ void __launch_bounds__(128, 1) k_mlp_infer(int n, const __nv_bfloat16* __restrict__ feat, MlpDev net,
                                                      float* __restrict__ out, int* err, int stall) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int fail;
    unsigned char* sm = smem_base(smem_raw);
    float* vec = reinterpret_cast<float*>(sm + SM_VEC);
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) {
        tc_alloc(&tmem_base, 128);
        tc_relinquish();
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        mbar_fence_init();
        fail = 0;
    }
    load_operand(sm + SM_W1, net.W1, MLP_H, MLP_IN);
    load_operand(sm + SM_W2, net.W2, MLP_H, MLP_H);
    load_vectors(vec, net);
    const float b3 = net.b3[0];
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = tmem_base;
    const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
    const uint32_t id64 = idesc_bf16(MLP_TILE, MLP_H);
    uint32_t phase = 0, fparity = 0;
    const int ntiles = (n + MLP_TILE - 1) / MLP_TILE;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int row = tile * MLP_TILE + tid;
        float x[16];
        load_x_row(sm, feat, n, row, tid, x);
        MLP_SYNC_ISSUE(tc_mma(tm + TM_D1, smem_desc(sm + SM_X, 128, 256), smem_desc(sm + SM_W1, 128, 256), id64, 0));
        // H1 = relu(D1 + b1) -> BF16 operand
#pragma unroll
        for (int c0 = 0; c0 < MLP_H; c0 += 16) {
            float v[16];
            tc_ld16(tm + lane_off + TM_D1 + c0, v);
            tc_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) v[q] = fmaxf(v[q] + vec[c0 + q], 0.f);
            st_row8(sm + SM_H1, tid, c0, MLP_H, v);
            st_row8(sm + SM_H1, tid, c0 + 8, MLP_H, v + 8);
        }
        MLP_SYNC_ISSUE(for (int kk = 0; kk < MLP_H / 16; kk++) tc_mma(
            tm + TM_D2, smem_desc(sm + SM_H1 + kk * 256, 128, 1024), smem_desc(sm + SM_W2 + kk * 256, 128, 1024),
            id64, kk > 0));
        // y = relu(D2 + b2) . w3 + b3
        float y = b3;
#pragma unroll
        for (int c0 = 0; c0 < MLP_H; c0 += 16) {
            float v[16];
            tc_ld16(tm + lane_off + TM_D2 + c0, v);
            tc_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) y += fmaxf(v[q] + vec[MLP_H + c0 + q], 0.f) * vec[2 * MLP_H + c0 + q];
        }
        if (row < n) out[row] = fail ? 0.f : y;
        tc_fence_before();
        __syncthreads();
        if (fail) break;
    }
    if (tid == 0 && fail) atomicOr(err, 1);
    MLP_DRAIN();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tc_dealloc(tmem_base, 128);
    }
}

// ---- gradient ---------------------------------------------------------------
// Loss L = sum_i w_i (y_i - t_i)^2 / sum_i w_i over the rows i < n
// (inv_wsum = 1 / sum_i w_i).  Writes this CTA's partial gradient
// (flattened like the parameters), sum w e^2 and sum w into
// part[blockIdx.x][MLP_PART].  The bias gradients come out of the
// weight-gradient MMAs through a row of ones appended to H1^T and X^T.
// Rounding points (kept by the oracle): H1, delta2 and delta1 are BF16 where
// an MMA reads them; the masks, y and dL/dy are FP32.
__global__ void __launch_bounds__(128, 1) k_mlp_grad(int n, const __nv_bfloat16* __restrict__ feat,
                                                     const float* __restrict__ target,
                                                     const float* __restrict__ weight, float inv_wsum, MlpDev net,
                                                     float* __restrict__ part, int* err) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int fail;
    __shared__ float red[4][MLP_H + 4];
    unsigned char* sm = smem_base(smem_raw);
    float* vec = reinterpret_cast<float*>(sm + SM_VEC);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        tc_alloc(&tmem_base, 256);
        tc_relinquish();
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        mbar_fence_init();
        fail = 0;
    }
    load_operand(sm + SM_W1, net.W1, MLP_H, MLP_IN);
    load_operand(sm + SM_W2, net.W2, MLP_H, MLP_H);
    load_operand(sm + SM_W2T, net.W2T, MLP_H, MLP_H);
    load_vectors(vec, net);
    // rows that stay zero: delta^T padding (64..127), H1^T 65..79, X^T 17..31
    for (int q = tid; q < 64 * 16; q += blockDim.x) {
        int r = 64 + q / 16, k0 = (q % 16) * 8;
        *reinterpret_cast<uint4*>(sm + SM_D2T + cm_off(r, k0, 128)) = make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4*>(sm + SM_D1T + cm_off(r, k0, 128)) = make_uint4(0, 0, 0, 0);
    }
    for (int q = tid; q < 15 * 16; q += blockDim.x) {
        int r = q / 16, k0 = (q % 16) * 8;
        *reinterpret_cast<uint4*>(sm + SM_H1T + cm_off(65 + r, k0, 128)) = make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4*>(sm + SM_XT + cm_off(17 + r, k0, 128)) = make_uint4(0, 0, 0, 0);
    }
    const float b3 = net.b3[0];
    float gw3[MLP_H];
#pragma unroll
    for (int c = 0; c < MLP_H; c++) gw3[c] = 0.f;
    float gb3 = 0.f, lsum = 0.f, wsum = 0.f;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = tmem_base;
    const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
    const uint32_t id64 = idesc_bf16(MLP_TILE, MLP_H), idw2 = idesc_bf16(MLP_TILE, GW2_N),
                   idw1 = idesc_bf16(MLP_TILE, GW1_N);
    uint32_t phase = 0, fparity = 0;
    const int stall = 0;
    int first = 1;
    const int ntiles = (n + MLP_TILE - 1) / MLP_TILE;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int row = tile * MLP_TILE + tid;
        const bool valid = row < n;
        float x[16];
        load_x_row(sm, feat, n, row, tid, x);
#pragma unroll
        for (int q = 0; q < 16; q++) st_bf16(sm + SM_XT, q, tid, 128, x[q]);
        st_bf16(sm + SM_XT, 16, tid, 128, valid ? 1.f : 0.f);
        st_bf16(sm + SM_H1T, 64, tid, 128, valid ? 1.f : 0.f);
        const float wi = valid ? weight[row] : 0.f, ti = valid ? target[row] : 0.f;
        MLP_SYNC_ISSUE(tc_mma(tm + TM_D1, smem_desc(sm + SM_X, 128, 256), smem_desc(sm + SM_W1, 128, 256), id64, 0));
        uint32_t m1lo = 0, m1hi = 0;   // ReLU masks of layer 1 (bit c: z1_c > 0)
#pragma unroll
        for (int c0 = 0; c0 < MLP_H; c0 += 16) {
            float v[16];
            tc_ld16(tm + lane_off + TM_D1 + c0, v);
            tc_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int c = c0 + q;
                float z = v[q] + vec[c];
                bool on = z > 0.f;
                if (on) {
                    if (c < 32) m1lo |= 1u << c;
                    else m1hi |= 1u << (c - 32);
                }
                v[q] = on ? z : 0.f;
                st_bf16(sm + SM_H1T, c, tid, 128, v[q]);
            }
            st_row8(sm + SM_H1, tid, c0, MLP_H, v);
            st_row8(sm + SM_H1, tid, c0 + 8, MLP_H, v + 8);
        }
        MLP_SYNC_ISSUE(for (int kk = 0; kk < MLP_H / 16; kk++) tc_mma(
            tm + TM_D2, smem_desc(sm + SM_H1 + kk * 256, 128, 1024), smem_desc(sm + SM_W2 + kk * 256, 128, 1024),
            id64, kk > 0));
        // y (first read of D2), then dL/dy, w3 gradient and delta2 (second read)
        float y = b3;
#pragma unroll
        for (int c0 = 0; c0 < MLP_H; c0 += 16) {
            float v[16];
            tc_ld16(tm + lane_off + TM_D2 + c0, v);
            tc_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) y += fmaxf(v[q] + vec[MLP_H + c0 + q], 0.f) * vec[2 * MLP_H + c0 + q];
        }
        const float e = y - ti;
        const float g3 = 2.f * wi * e * inv_wsum;
        lsum += wi * e * e;
        wsum += wi;
        gb3 += g3;
#pragma unroll
        for (int c0 = 0; c0 < MLP_H; c0 += 16) {
            float v[16];
            tc_ld16(tm + lane_off + TM_D2 + c0, v);
            tc_wait_ld();
#pragma unroll
            for (int h = 0; h < 16; h += 8) {
                float d[8];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int c = c0 + h + q;
                    float h2 = fmaxf(v[h + q] + vec[MLP_H + c], 0.f);
                    gw3[c] += g3 * h2;
                    d[q] = h2 > 0.f ? g3 * vec[2 * MLP_H + c] : 0.f;
                    st_bf16(sm + SM_D2T, c, tid, 128, d[q]);
                }
                st_row8(sm + SM_D2, tid, c0 + h, MLP_H, d);
            }
        }
        // D3 = delta2 W2 (B operand W2^T); [dW2 | db2] += delta2^T [H1 | 1]
        MLP_SYNC_ISSUE({
            for (int kk = 0; kk < MLP_H / 16; kk++)
                tc_mma(tm + TM_D1, smem_desc(sm + SM_D2 + kk * 256, 128, 1024),
                       smem_desc(sm + SM_W2T + kk * 256, 128, 1024), id64, kk > 0);
            for (int kk = 0; kk < MLP_TILE / 16; kk++)
                tc_mma(tm + TM_GW2, smem_desc(sm + SM_D2T + kk * 256, 128, 2048),
                       smem_desc(sm + SM_H1T + kk * 256, 128, 2048), idw2, (first == 0 || kk > 0));
        });
        // delta1 = D3 (z1 > 0)
#pragma unroll
        for (int c0 = 0; c0 < MLP_H; c0 += 16) {
            float v[16];
            tc_ld16(tm + lane_off + TM_D1 + c0, v);
            tc_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int c = c0 + q;
                bool on = (c < 32) ? ((m1lo >> c) & 1u) : ((m1hi >> (c - 32)) & 1u);
                st_bf16(sm + SM_D1T, c, tid, 128, on ? v[q] : 0.f);
            }
        }
        // [dW1 | db1] += delta1^T [X | 1]
        MLP_SYNC_ISSUE(for (int kk = 0; kk < MLP_TILE / 16; kk++) tc_mma(
            tm + TM_GW1, smem_desc(sm + SM_D1T + kk * 256, 128, 2048), smem_desc(sm + SM_XT + kk * 256, 128, 2048),
            idw1, (first == 0 || kk > 0)));
        first = 0;
        tc_fence_before();
        __syncthreads();
        if (fail) break;
    }
    // this CTA's partial gradient
    float* P = part + (size_t)blockIdx.x * MLP_PART;
    tc_fence_after();
    if (warp < 2) {
        const int u = tid;   // TMEM lane = unit
        if (!first && !fail) {
#pragma unroll
            for (int c0 = 0; c0 < MLP_H; c0 += 16) {
                float v[16];
                tc_ld16(tm + lane_off + TM_GW2 + c0, v);
                tc_wait_ld();
#pragma unroll
                for (int q = 0; q < 16; q++) P[MLP_OFF_W2 + u * MLP_H + c0 + q] = v[q];
            }
            float v[16];
            tc_ld16(tm + lane_off + TM_GW2 + MLP_H, v);
            tc_wait_ld();
            P[MLP_OFF_B2 + u] = v[0];
            tc_ld16(tm + lane_off + TM_GW1, v);
            tc_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) P[MLP_OFF_W1 + u * MLP_IN + q] = v[q];
            tc_ld16(tm + lane_off + TM_GW1 + 16, v);
            tc_wait_ld();
            P[MLP_OFF_B1 + u] = v[0];
        } else {
            for (int q = 0; q < MLP_H; q++) P[MLP_OFF_W2 + u * MLP_H + q] = 0.f;
            for (int q = 0; q < MLP_IN; q++) P[MLP_OFF_W1 + u * MLP_IN + q] = 0.f;
            P[MLP_OFF_B2 + u] = 0.f;
            P[MLP_OFF_B1 + u] = 0.f;
        }
    } else if (warp >= 2) {
        // warps 2, 3 idle in the TMEM read-out: their lanes hold padding rows
    }
    // w3 gradient: warp shuffles, then the 4 warps in order
#pragma unroll
    for (int c = 0; c < MLP_H; c++) {
        float d = gw3[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) red[warp][c] = d;
    }
    float s3 = gb3, sl = lsum, sw = wsum;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s3 += __shfl_xor_sync(0xffffffffu, s3, o);
        sl += __shfl_xor_sync(0xffffffffu, sl, o);
        sw += __shfl_xor_sync(0xffffffffu, sw, o);
    }
    if (lane == 0) {
        red[warp][MLP_H] = s3;
        red[warp][MLP_H + 1] = sl;
        red[warp][MLP_H + 2] = sw;
    }
    __syncthreads();
    for (int c = tid; c < MLP_H + 3; c += blockDim.x) {
        float s = red[0][c] + red[1][c] + red[2][c] + red[3][c];
        if (c < MLP_H) P[MLP_OFF_W3 + c] = s;
        else if (c == MLP_H) P[MLP_OFF_B3] = s;
        else if (c == MLP_H + 1) P[MLP_NPARAM] = s;
        else P[MLP_NPARAM + 1] = s;
    }
    if (tid == 0 && fail) atomicOr(err, 1);
    MLP_DRAIN();
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tc_dealloc(tmem_base, 256);
    }
}

// ---- Adam step on the FP32 master parameters -----------------------------------
// grad = sum over the CTA partials in CTA order; refresh the BF16 copies.
struct MlpOpt {
    float *master, *m, *v;     // MLP_NPARAM each
    __nv_bfloat16 *W1, *W2, *W2T;
    float *b1, *b2, *w3, *b3;
    float* loss;               // [sum w e^2, sum w] of the last gradient pass
    const double* tstep;       // Adam step number on the device (nullptr: the argument t)
};

__global__ void k_mlp_adam(int nparts, const float* __restrict__ part, MlpOpt o, float lr, float beta1,
                           float beta2, float eps, int t, int apply) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < MLP_NPARAM + 2; p += gridDim.x * blockDim.x) {
        float g = 0.f;
        for (int c = 0; c < nparts; c++) g += part[(size_t)c * MLP_PART + p];
        if (p >= MLP_NPARAM) {
            if (p == MLP_NPARAM) o.loss[0] = g;   // sum w e^2 (divided by the weight sum on the host)
            else o.loss[1] = g;
            continue;
        }
        float w = o.master[p];
        if (apply) {
            float m = beta1 * o.m[p] + (1.f - beta1) * g;
            float v = beta2 * o.v[p] + (1.f - beta2) * g * g;
            o.m[p] = m;
            o.v[p] = v;
            float tt = o.tstep ? (float)o.tstep[0] : (float)t;
            float mh = m / (1.f - powf(beta1, tt)), vh = v / (1.f - powf(beta2, tt));
            w -= lr * mh / (sqrtf(vh) + eps);
            o.master[p] = w;
        }
        __nv_bfloat16 wb = __float2bfloat16_rn(w);
        if (p < MLP_OFF_B1) {
            o.W1[p - MLP_OFF_W1] = wb;
        } else if (p < MLP_OFF_W2) {
            o.b1[p - MLP_OFF_B1] = w;
        } else if (p < MLP_OFF_B2) {
            int q = p - MLP_OFF_W2, r = q / MLP_H, c = q % MLP_H;
            o.W2[q] = wb;
            o.W2T[c * MLP_H + r] = wb;
        } else if (p < MLP_OFF_W3) {
            o.b2[p - MLP_OFF_B2] = w;
        } else if (p < MLP_OFF_B3) {
            o.w3[p - MLP_OFF_W3] = __bfloat162float(wb);
        } else {
            o.b3[0] = w;
        }
    }
}

}  // namespace sphdem
