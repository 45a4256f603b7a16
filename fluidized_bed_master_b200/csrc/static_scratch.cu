// static_scratch.cu -- allocation-free variant of the NNPS cell sort.
//
// sphdem_sort_cells_static does what the engine's NNPS does at the start of
// every step (cell key per particle, stable sort by cell, cell start/end),
// but it never allocates device memory: its scratch (unsorted keys, slot
// indices and the radix-sort workspace) lives in one file-scope
// __device__ array of SPHDEM_STATIC_SCRATCH_BYTES.  It exists for callers
// that must not allocate once their time loop runs: a host application that
// hands all device memory out of its own pool and forbids allocations after
// start-up (its footprint is fixed when the run starts), or a coupled solver
// whose other streams must not stall, since cudaMalloc and cudaFree may
// synchronise the whole device.
//
// Every GPU that loads the library holds the array until the process exits.
// All calls on a device share it, so calls that overlap on the GPU (two
// streams, two host threads) race; the array keeps the previous call's
// contents, and everything the kernels read from it is written first in
// the same call.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/sphdem.h"
#include "device_common.cuh"

namespace {

constexpr size_t kScratchBytes = SPHDEM_STATIC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
// the two key/slot arrays of the largest call must leave room for the sort's workspace
static_assert(2 * (((size_t)SPHDEM_STATIC_MAX_PARTICLES * sizeof(int) + 255) & ~(size_t)255) < kScratchBytes,
              "SPHDEM_STATIC_MAX_PARTICLES does not fit SPHDEM_STATIC_SCRATCH_BYTES");

__device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

// device address of g_sort_scratch per device, resolved once with that device current
void* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

int scratch_for_current_device(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SPHDEM_E_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return SPHDEM_E_ARG;
    std::lock_guard<std::mutex> lk(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || !p) return SPHDEM_E_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return SPHDEM_OK;
}

// cell key of KERNEL_index_particle_to_cell_* (functions_NNPS.cuh:762-821)
__global__ void k_static_hash(sphdem::DevParams P, int n, const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, int* key, int* val) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int ic, jc, kc;
    sphdem::cell_ijk(P, x[i], y[i], z[i], ic, jc, kc);
    key[i] = ic + P.NI * jc + P.NI * P.NJ * kc;
    val[i] = i;
}

// cell start/end of KERNEL_reorder_* (functions_NNPS.cuh:670-730)
__global__ void k_static_bounds(int n, const int* __restrict__ key, int* start, int* end) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = key[i];
    if (i == 0 || k != key[i - 1]) {
        start[k] = i;
        if (i > 0) end[key[i - 1]] = i;
    }
    if (i == n - 1) end[k] = n;
}

}  // namespace

extern "C" int sphdem_sort_cells_static(const double* x, const double* y, const double* z, int32_t n,
                                        const double* bbox, const int32_t* nijk, int32_t* perm, int32_t* cell_key,
                                        int32_t* cell_start, int32_t* cell_end, void* stream) {
    if (!x || !y || !z || !bbox || !nijk || !perm || !cell_key || !cell_start || !cell_end || n < 0)
        return SPHDEM_E_ARG;
    if (n > SPHDEM_STATIC_MAX_PARTICLES) return SPHDEM_E_NOMEM;
    if (nijk[0] <= 0 || nijk[1] <= 0 || nijk[2] <= 0) return SPHDEM_E_ARG;
    long long ncells = (long long)nijk[0] * nijk[1] * nijk[2];
    if (ncells > (1ll << 30)) return SPHDEM_E_NOMEM;
    cudaStream_t st = (cudaStream_t)stream;
    // empty cells read -1 (cu_memset, Variable_Type.cuh)
    if (cudaMemsetAsync(cell_start, 0xff, sizeof(int32_t) * ncells, st) != cudaSuccess) return SPHDEM_E_CUDA;
    if (n == 0) return SPHDEM_OK;
    void* base = nullptr;
    int r = scratch_for_current_device(&base);
    if (r) return r;
    // carve: unsorted keys | slot indices | radix-sort workspace (256-B aligned)
    size_t kbytes = ((size_t)n * sizeof(int) + 255) & ~(size_t)255;
    int* key_in = (int*)base;
    int* val_in = (int*)((char*)base + kbytes);
    void* tmp = (char*)base + 2 * kbytes;
    if (2 * kbytes >= kScratchBytes) return SPHDEM_E_NOMEM;
    size_t tmp_cap = kScratchBytes - 2 * kbytes;
    int bits = 1;
    while ((1ll << bits) <= ncells) bits++;
    size_t need = 0;
    if (cub::DeviceRadixSort::SortPairs(nullptr, need, key_in, cell_key, val_in, perm, n, 0, bits, st) != cudaSuccess)
        return SPHDEM_E_CUDA;
    if (need > tmp_cap) return SPHDEM_E_NOMEM;
    sphdem::DevParams P;
    memset(&P, 0, sizeof(P));
    P.NI = nijk[0]; P.NJ = nijk[1]; P.NK = nijk[2];
    P.num_cells = (int)ncells + 1;
    P.xmin = bbox[0]; P.xmax = bbox[1]; P.ymin = bbox[2]; P.ymax = bbox[3]; P.zmin = bbox[4]; P.zmax = bbox[5];
    const int tpb = 128;
    int blocks = (n + tpb - 1) / tpb;
    k_static_hash<<<blocks, tpb, 0, st>>>(P, n, x, y, z, key_in, val_in);
    if (cudaGetLastError() != cudaSuccess) return SPHDEM_E_CUDA;
    if (cub::DeviceRadixSort::SortPairs(tmp, need, key_in, cell_key, val_in, perm, n, 0, bits, st) != cudaSuccess)
        return SPHDEM_E_CUDA;
    k_static_bounds<<<blocks, tpb, 0, st>>>(n, cell_key, cell_start, cell_end);
    if (cudaGetLastError() != cudaSuccess) return SPHDEM_E_CUDA;
    return SPHDEM_OK;
}
