// host_shim.h -- TEST INFRASTRUCTURE ONLY.
//
// Lets the reference's CUDA C++ (SOPHIA_gpu.cu and its headers, after the
// mechanical rewrite in oracle/Makefile's `refhost` recipe) compile with a
// host C++ compiler, so that the reference's own per-particle kernel bodies
// run on the CPU cores, looped with OpenMP.  It is force-included
// (g++ -include host_shim.h) ahead of the reference sources and provides:
//   * the CUDA qualifiers as no-ops (__global__/__device__/__host__/
//     __constant__), so kernels and device functions become host functions
//     and __constant__ tables become host globals;
//   * threadIdx/blockIdx/blockDim/gridDim as per-OS-thread variables, and
//     launch_host(), which replaces every `K<<<grid, block, ...>>>(args)`:
//     the grid's blocks are spread over OpenMP threads (dynamic schedule),
//     and a block's threads run one after another in threadIdx order;
//   * the CUDA runtime calls the reference makes (memory, copies, symbols,
//     streams, errors) as host memory operations;
//   * cub::DeviceRadixSort::SortPairs as a stable sort by key (CUB's radix
//     sort is stable, so the permutation is the same) and
//     cub::DeviceReduce::Max as a sequential maximum.
// Running a block's threads in order is exact for every kernel the ISPH-DEM
// step launches: the only ones that synchronise a block (KERNEL_reorder*,
// functions_NNPS.cuh:641-730) read, after their one __syncthreads, only the
// shared slot that the next-lower thread wrote before it, so __syncthreads
// is a no-op here and the dynamic shared array is a per-OS-thread buffer.
#pragma once

#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <type_traits>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline
#define __launch_bounds__(...)

struct dim3 {
    unsigned x, y, z;
    dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
struct uint3_host {
    unsigned x, y, z;
};

extern thread_local uint3_host host_threadIdx, host_blockIdx;
extern thread_local dim3 host_blockDim, host_gridDim;
#define threadIdx host_threadIdx
#define blockIdx host_blockIdx
#define blockDim host_blockDim
#define gridDim host_gridDim

inline void __syncthreads() {}

// per-OS-thread buffer that stands for a block's dynamic shared memory
int* host_shared_ints();

// CUDA's min/max on mixed int/floating arguments promote to the floating
// type (fmin/fmax: a NaN argument yields the other one)
template <class A, class B>
inline typename std::common_type<A, B>::type min(A a, B b) {
    typedef typename std::common_type<A, B>::type T;
    if (std::is_floating_point<T>::value) return (T)std::fmin((double)a, (double)b);
    return (T)a < (T)b ? (T)a : (T)b;
}
template <class A, class B>
inline typename std::common_type<A, B>::type max(A a, B b) {
    typedef typename std::common_type<A, B>::type T;
    if (std::is_floating_point<T>::value) return (T)std::fmax((double)a, (double)b);
    return (T)a > (T)b ? (T)a : (T)b;
}
using std::abs;
using std::fabs;
using std::floor;
using std::pow;
using std::sqrt;

// ---- runtime ------------------------------------------------------------
typedef int cudaError_t;
typedef void* cudaStream_t;
typedef void* cudaEvent_t;
enum { cudaSuccess = 0, cudaErrorHost = 1 };
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost,
                      cudaMemcpyDeviceToDevice, cudaMemcpyDefault };
struct cudaDeviceProp {
    char name[256];
    size_t totalGlobalMem, totalConstMem, sharedMemPerBlock, memPitch, textureAlignment;
    int major, minor, multiProcessorCount, clockRate, regsPerBlock, warpSize, maxThreadsPerBlock;
    int maxThreadsDim[3], maxGridSize[3];
    int deviceOverlap, kernelExecTimeoutEnabled, integrated, canMapHostMemory, computeMode;
    int memoryClockRate, memoryBusWidth, l2CacheSize, maxThreadsPerMultiProcessor;
};
inline const char* cudaGetErrorString(cudaError_t) { return "host"; }
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline cudaError_t cudaPeekAtLastError() { return cudaSuccess; }
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaThreadSynchronize() { return cudaSuccess; }
inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
inline cudaError_t cudaGetDevice(int* d) { *d = 0; return cudaSuccess; }
inline cudaError_t cudaGetDeviceCount(int* n) { *n = 1; return cudaSuccess; }
inline cudaError_t cudaDeviceReset() { return cudaSuccess; }
inline cudaError_t cudaGetDeviceProperties(cudaDeviceProp* p, int) {
    memset(p, 0, sizeof(*p));
    strcpy(p->name, "host");
    return cudaSuccess;
}
inline cudaError_t cudaDeviceCanAccessPeer(int* c, int, int) { *c = 0; return cudaSuccess; }
inline cudaError_t cudaDeviceEnablePeerAccess(int, unsigned) { return cudaSuccess; }
inline cudaError_t cudaDeviceDisablePeerAccess(int) { return cudaSuccess; }
inline cudaError_t cudaStreamCreate(cudaStream_t* s) { *s = nullptr; return cudaSuccess; }
inline cudaError_t cudaStreamDestroy(cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaEventCreate(cudaEvent_t* e) { *e = nullptr; return cudaSuccess; }
inline cudaError_t cudaEventRecord(cudaEvent_t, cudaStream_t = nullptr) { return cudaSuccess; }
inline cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
inline cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t, cudaEvent_t) { *ms = 0; return cudaSuccess; }
inline cudaError_t cudaEventDestroy(cudaEvent_t) { return cudaSuccess; }
inline cudaError_t cudaMalloc(void** p, size_t n) {
    *p = calloc(n ? n : 1, 1);
    return *p ? cudaSuccess : cudaErrorHost;
}
template <class T>
inline cudaError_t cudaMalloc(T** p, size_t n) { return cudaMalloc((void**)p, n); }
inline cudaError_t cudaMallocHost(void** p, size_t n) { return cudaMalloc(p, n); }
template <class T>
inline cudaError_t cudaMallocHost(T** p, size_t n) { return cudaMalloc((void**)p, n); }
inline cudaError_t cudaFree(void* p) { free(p); return cudaSuccess; }
inline cudaError_t cudaFreeHost(void* p) { free(p); return cudaSuccess; }
inline cudaError_t cudaMemset(void* p, int v, size_t n) { memset(p, v, n); return cudaSuccess; }
inline cudaError_t cudaMemsetAsync(void* p, int v, size_t n, cudaStream_t = nullptr) { memset(p, v, n); return cudaSuccess; }
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
    if (n) memmove(d, s, n);
    return cudaSuccess;
}
inline cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind k, cudaStream_t = nullptr) {
    return cudaMemcpy(d, s, n, k);
}
inline cudaError_t cudaMemcpyPeer(void* d, int, const void* s, int, size_t n) {
    return cudaMemcpy(d, s, n, cudaMemcpyDefault);
}
inline cudaError_t cudaMemcpyPeerAsync(void* d, int, const void* s, int, size_t n, cudaStream_t = nullptr) {
    return cudaMemcpy(d, s, n, cudaMemcpyDefault);
}
template <class T>
inline cudaError_t cudaMemcpyToSymbol(T& sym, const void* src, size_t n, size_t off = 0,
                                      cudaMemcpyKind = cudaMemcpyHostToDevice) {
    memcpy((char*)&sym + off, src, n);
    return cudaSuccess;
}
template <class T>
inline cudaError_t cudaMemcpyFromSymbol(void* dst, const T& sym, size_t n, size_t off = 0,
                                        cudaMemcpyKind = cudaMemcpyDeviceToHost) {
    memcpy(dst, (const char*)&sym + off, n);
    return cudaSuccess;
}

// ---- kernel launch --------------------------------------------------------
struct LaunchCfg {
    dim3 grid, block;
    LaunchCfg(dim3 g, dim3 b, size_t = 0, cudaStream_t = nullptr) : grid(g), block(b) {}
};

template <class F, class... A>
inline void launch_host(LaunchCfg c, F&& kern, A... args) {
    const long nb = (long)c.grid.x * c.grid.y * c.grid.z;
#pragma omp parallel for schedule(dynamic, 8)
    for (long b = 0; b < nb; b++) {
        host_gridDim = c.grid;
        host_blockDim = c.block;
        host_blockIdx.x = (unsigned)(b % c.grid.x);
        host_blockIdx.y = (unsigned)((b / c.grid.x) % c.grid.y);
        host_blockIdx.z = (unsigned)(b / ((long)c.grid.x * c.grid.y));
        for (unsigned tz = 0; tz < c.block.z; tz++)
            for (unsigned ty = 0; ty < c.block.y; ty++)
                for (unsigned tx = 0; tx < c.block.x; tx++) {
                    host_threadIdx.x = tx;
                    host_threadIdx.y = ty;
                    host_threadIdx.z = tz;
                    kern(args...);
                }
    }
}

// ---- CUB ------------------------------------------------------------------
namespace cub {
struct DeviceRadixSort {
    template <class K, class V>
    static cudaError_t SortPairs(void* tmp, size_t& bytes, const K* kin, K* kout, const V* vin, V* vout, int n,
                                 int = 0, int = (int)(sizeof(K) * 8), cudaStream_t = nullptr, bool = false) {
        if (!tmp) {
            bytes = 16;
            return cudaSuccess;
        }
        std::vector<int> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [kin](int a, int b) { return kin[a] < kin[b]; });
        std::vector<K> k2(n);
        std::vector<V> v2(n);
        for (int i = 0; i < n; i++) {
            k2[i] = kin[ord[i]];
            v2[i] = vin[ord[i]];
        }
        std::copy(k2.begin(), k2.end(), kout);
        std::copy(v2.begin(), v2.end(), vout);
        return cudaSuccess;
    }
};
struct DeviceReduce {
    template <class I, class O>
    static cudaError_t Max(void* tmp, size_t& bytes, I in, O out, int n, cudaStream_t = nullptr, bool = false) {
        if (!tmp) {
            bytes = 16;
            return cudaSuccess;
        }
        auto m = in[0];
        for (int i = 1; i < n; i++)
            if (m < in[i]) m = in[i];
        *out = m;
        return cudaSuccess;
    }
};
}  // namespace cub
