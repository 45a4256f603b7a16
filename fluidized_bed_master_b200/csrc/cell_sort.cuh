// cell_sort.cuh -- the NNPS sort by cell, written for this engine.
//
// Replaces cub::DeviceRadixSort::SortPairs of the reference's NNPS
// (ISPH_Calc_seperate.cuh:83-85, WCSPH_Calc.cuh:36) and the cell start/end
// search of KERNEL_reorder_* (functions_NNPS.cuh:670-730).  The values are
// the slot indices 0..n-1 and CUB's radix sort is stable, so the reference's
// permutation is: keys ascending, equal keys in ascending slot order.  A
// counting sort gives exactly that with one pass over the keys per phase:
//
//   count   fused into the hash kernels (cell_count): cnt[key] += 1, one
//           atomic per distinct key of a warp (__match_any_sync);
//   scan    k_sort_tile_sums + k_sort_scan: exclusive prefix of cnt over the
//           ncell + 1 buckets (the last bucket holds the i_type 3 slots that
//           the reference keys num_cells) -> start[]; resets fill[];
//   scatter k_sort_scatter: tmp[start[k] + fill[k]++] = slot, one atomic
//           per distinct key of a warp; order inside a cell is arbitrary;
//   settle  k_sort_settle, one warp per bucket (per 32 buckets on a sparse
//           grid, cell_sort_sparse): ranks the bucket's slots by
//           value (unique, so ranks are a permutation), writes perm/key in
//           ascending slot order, the cell's start (-1 when empty) and end,
//           and zeroes cnt[] for the next step.
//
// Every bucket is owned by one warp in the settle pass and the ranks depend
// only on the values, so the result is deterministic and bit-identical to
// CUB's.  No memset runs per step: cnt is zeroed by the settle pass, fill by
// the scan (both start at zero after allocation).
//
// The warp's ranking costs m^2/32 for a bucket of m slots: fine for cells
// (tens of particles), not for a last bucket holding the many parked spare
// slots of a slab of a sharded bed.  With `big_last` set, that bucket is
// written instead by a stable compaction of the slots keyed num_cells
// (block counts, one-block scan, ordered writes): the same ascending order.
#pragma once
#include <climits>
#include <cuda_runtime.h>

namespace sphdem {

// Programmatic dependent launch (launch_pdl in engine.cu): a kernel launched
// with programmatic stream serialization may be scheduled while the previous
// kernel of its stream drains, and waits here, before touching memory, until
// that kernel has completed and its writes are visible (a no-op for a plain
// launch).  Every thread waits before any early return, so a kernel never
// completes before its predecessor: the chain stays transitive.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// launch with programmatic stream serialization: the kernel may be
// scheduled while its stream's previous kernel drains (it must begin with
// grid_dep_wait).  Inside a captured graph this becomes a programmatic edge.
template <typename... KP, typename... A>
inline cudaError_t launch_pdl(void (*k)(KP...), dim3 g, dim3 b, size_t smem, cudaStream_t st, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = g;
    cfg.blockDim = b;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

constexpr int SORT_TILE = 4096;   // scan tile: 1024 threads x 4 buckets

struct CellSort {
    int* cnt;        // [nb] bucket counts (zero between steps)
    int* fill;       // [nb] scatter cursors
    int* start;      // [nb] exclusive prefix of cnt
    int* tile_sum;   // [ntiles]
    int* tmp;        // [n] slots grouped by bucket, unordered inside a bucket
    int nb;          // buckets: num_cells + 1
    int ntiles;
    int big_last;    // the last bucket by compaction (blk: per-block counts)
    int* blk;
    // On a sparse grid (cell_sort_sparse), the occupied cells (< nb - 1) in
    // no particular order and their count, for the passes that take a warp
    // per cell; null when not kept.
    int* occ = nullptr;
    int* occ_n = nullptr;
};

// A sparse grid (e.g. 2-D beds in planes): the settle pass takes 32 buckets
// per warp and, where the sort keeps the list, lists the occupied cells.
// Sparse means more cells than keys / 4 for a sort that lists its occupied
// cells (the SPH set, whose warp-per-cell passes then skip the empty
// cells), else more than twice as many cells as keys.
inline bool cell_sort_sparse(const CellSort& cs, int n) { return cs.occ ? 4ll * cs.nb > n : cs.nb > 2ll * n; }

// count one key (called by every thread of a warp that hashes; inactive
// threads pass key < 0)
__device__ __forceinline__ void cell_count(int* cnt, int key) {
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, key);
    const int lane = threadIdx.x & 31;
    if (key >= 0 && lane == __ffs(peers) - 1) atomicAdd(&cnt[key], __popc(peers));
}

__global__ void __launch_bounds__(1024) k_sort_tile_sums(const int* __restrict__ cnt, int nb, int* tile_sum,
                                                         int* occ_n) {
    grid_dep_wait();
    if (occ_n && blockIdx.x == 0 && threadIdx.x == 0) *occ_n = 0;   // refilled by the settle pass
    const int base = blockIdx.x * SORT_TILE + threadIdx.x * 4;
    int s = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) s += (base + q < nb) ? cnt[base + q] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ int ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        int v = ws[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) tile_sum[blockIdx.x] = v;
    }
}

// start[b] = sum of cnt[0..b); the tile's offset is the sum of the earlier
// tiles' sums (in tile order); fill[] is reset for the scatter
__global__ void __launch_bounds__(1024) k_sort_scan(const int* __restrict__ cnt, const int* __restrict__ tile_sum,
                                                    int nb, int* start, int* fill) {
    grid_dep_wait();
    __shared__ int ws[32];
    __shared__ int toff;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
        int acc = 0;
        for (int t0 = 0; t0 < (int)blockIdx.x; t0 += 32) {
            int v = (t0 + lane < (int)blockIdx.x) ? tile_sum[t0 + lane] : 0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            acc += v;
        }
        if (lane == 0) toff = acc;
    }
    const int base = blockIdx.x * SORT_TILE + threadIdx.x * 4;
    int c[4], s = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        c[q] = (base + q < nb) ? cnt[base + q] : 0;
        s += c[q];
    }
    // inclusive warp scan of the thread sums
    int inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int v = ws[lane], w = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        ws[lane] = w - v;   // exclusive prefix of the warp totals
    }
    __syncthreads();
    int run = toff + ws[warp] + inc - s;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (base + q < nb) {
            start[base + q] = run;
            fill[base + q] = 0;
        }
        run += c[q];
    }
}

__global__ void k_sort_scatter(int n, const int* __restrict__ key, const int* __restrict__ start, int* fill,
                               int* tmp) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = i < n ? key[i] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, k);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (k >= 0 && lane == leader) base = atomicAdd(&fill[k], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (k >= 0) tmp[start[k] + base + __popc(peers & ((1u << lane) - 1u))] = i;
}

// the ranking of one bucket of m >= 2 slots from s by a warp
__device__ __forceinline__ void settle_bucket(int b, int m, int s, const int* __restrict__ tmp, int* perm,
                                              int* key_out, int lane) {
    for (int a = 0; a < m; a += 32) {
        const int v = (a + lane < m) ? tmp[s + a + lane] : INT_MAX;
        int r = 0;
        for (int a2 = 0; a2 < m; a2 += 32) {
            const int w0 = (a2 + lane < m) ? tmp[s + a2 + lane] : INT_MAX;
#pragma unroll
            for (int j = 0; j < 32; j++) r += (__shfl_sync(0xffffffffu, w0, j) < v);
        }
        if (a + lane < m) {
            perm[s + r] = v;
            key_out[s + r] = b;
        }
    }
}

// G buckets per warp (G = 1, or 32 for a grid of mostly empty cells): lane
// l < G owns bucket b = warp * G + l; cell b < nb - 1 gets gs (start or -1)
// and ge (end, written only for a non-empty cell, as the reference's reorder
// does).  A bucket of one slot is settled by its lane; the warp ranks the
// buckets of two or more slots one after another.
template <int G>
__global__ void __launch_bounds__(256) k_sort_settle(int nb, int* cnt, const int* __restrict__ start,
                                                     const int* __restrict__ tmp, int* perm, int* key_out, int* gs,
                                                     int* ge, int skip_last, int* occ, int* occ_n) {
    grid_dep_wait();
    const int b0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * G;
    const int lane = threadIdx.x & 31;
    if (b0 >= nb) return;
    const int bl = b0 + lane;
    const bool own = lane < G && bl < nb;
    const int ml = own ? cnt[bl] : 0;
    const int sl = own ? start[bl] : 0;
    __syncwarp();
    if (own) {
        if (ml) cnt[bl] = 0;
        if (bl < nb - 1) {
            gs[bl] = ml ? sl : -1;
            if (ml) ge[bl] = sl + ml;
        }
        if (ml == 1 && !(skip_last && bl == nb - 1)) {
            perm[sl] = tmp[sl];
            key_out[sl] = bl;
        }
    }
    if (occ) {   // append the warp's occupied cells
        const bool oc = own && ml > 0 && bl < nb - 1;
        const unsigned om = __ballot_sync(0xffffffffu, oc);
        int base = 0;
        if (om && lane == 0) base = atomicAdd(occ_n, __popc(om));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (oc) occ[base + __popc(om & ((1u << lane) - 1u))] = bl;
    }
    unsigned multi = __ballot_sync(0xffffffffu, own && ml >= 2 && !(skip_last && bl == nb - 1));
    while (multi) {
        const int k = __ffs(multi) - 1;
        multi &= multi - 1;
        const int b = b0 + k, m = __shfl_sync(0xffffffffu, ml, k), s = __shfl_sync(0xffffffffu, sl, k);
        settle_bucket(b, m, s, tmp, perm, key_out, lane);
    }
}

// the last bucket (key last) by stable compaction: per-block counts ...
__global__ void __launch_bounds__(256) k_sort_last_count(int n, const int* __restrict__ key, int last, int* blk) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = __syncthreads_count(i < n && key[i] == last);
    if (threadIdx.x == 0) blk[blockIdx.x] = c;
}

// ... their exclusive prefix (one block of 1024 threads) ...
__global__ void __launch_bounds__(1024) k_sort_last_scan(int nblk, int* blk) {
    __shared__ int part[1024];
    const int per = (nblk + 1023) / 1024, b0 = threadIdx.x * per, b1 = min(nblk, b0 + per);
    int s = 0;
    for (int b = b0; b < b1; b++) s += blk[b];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int acc = part[threadIdx.x] - s;
    for (int b = b0; b < b1; b++) {
        const int v = blk[b];
        blk[b] = acc;
        acc += v;
    }
}

// ... and the slots in ascending order from the bucket's start
__global__ void __launch_bounds__(256) k_sort_last_write(int n, const int* __restrict__ key, int last,
                                                         const int* __restrict__ blk, const int* __restrict__ start,
                                                         int* perm, int* key_out) {
    __shared__ int wsum[8];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool f = i < n && key[i] == last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[w] = __popc(m);
    __syncthreads();
    int pos = start[last] + blk[blockIdx.x];
    for (int k = 0; k < w; k++) pos += wsum[k];
    if (f) {
        pos += __popc(m & ((1u << lane) - 1u));
        perm[pos] = i;
        key_out[pos] = last;
    }
}

// scan + scatter + settle for n keys already counted into cs.cnt
inline cudaError_t cell_sort(const CellSort& cs, int n, const int* key_in, int* perm, int* key_out, int* gs, int* ge,
                             cudaStream_t st) {
    cudaError_t e;
    const bool sparse = cell_sort_sparse(cs, n);
    int* occ_n = sparse ? cs.occ_n : nullptr;
    if ((e = launch_pdl(k_sort_tile_sums, cs.ntiles, 1024, 0, st, (const int*)cs.cnt, cs.nb, cs.tile_sum, occ_n)))
        return e;
    if ((e = launch_pdl(k_sort_scan, cs.ntiles, 1024, 0, st, (const int*)cs.cnt, (const int*)cs.tile_sum, cs.nb,
                        cs.start, cs.fill)))
        return e;
    if (n > 0 && (e = launch_pdl(k_sort_scatter, (n + 255) / 256, 256, 0, st, n, key_in, (const int*)cs.start,
                                 cs.fill, cs.tmp)))
        return e;
    const int big = cs.big_last && n > 0;
    // a grid of mostly empty cells (e.g. 2-D beds in planes): 32 buckets per warp
    if (sparse) {
        const int nw = (cs.nb + 31) / 32;
        if ((e = launch_pdl(k_sort_settle<32>, (nw * 32 + 255) / 256, 256, 0, st, cs.nb, cs.cnt,
                            (const int*)cs.start, (const int*)cs.tmp, perm, key_out, gs, ge, big,
                            occ_n ? cs.occ : (int*)nullptr, occ_n)))
            return e;
    } else if ((e = launch_pdl(k_sort_settle<1>, (cs.nb * 32 + 255) / 256, 256, 0, st, cs.nb, cs.cnt,
                               (const int*)cs.start, (const int*)cs.tmp, perm, key_out, gs, ge, big,
                               (int*)nullptr, (int*)nullptr))) {
        return e;
    }
    if (big) {
        const int nblk = (n + 255) / 256;
        k_sort_last_count<<<nblk, 256, 0, st>>>(n, key_in, cs.nb - 1, cs.blk);
        k_sort_last_scan<<<1, 1024, 0, st>>>(nblk, cs.blk);
        k_sort_last_write<<<nblk, 256, 0, st>>>(n, key_in, cs.nb - 1, cs.blk, cs.start, perm, key_out);
    }
    return cudaGetLastError();
}

}  // namespace sphdem
