// host_shim.cpp -- TEST INFRASTRUCTURE ONLY: the per-OS-thread launch
// indices and shared-memory buffer declared in host_shim.h.
#include "host_shim.h"

thread_local uint3_host host_threadIdx, host_blockIdx;
thread_local dim3 host_blockDim, host_gridDim;

// a block's dynamic shared memory: the reference launches its reorder
// kernels with (blockDim.x + 1) ints (functions_NNPS.cuh:641-730)
int* host_shared_ints() {
    static thread_local std::vector<int> buf;
    if (buf.size() < 4096) buf.resize(4096);
    return buf.data();
}
