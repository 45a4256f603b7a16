// mlp.cu -- host side of the learned PPE warm start network
// (mlp_tcgen05.cuh): device buffers, launches, and the C-ABI entry points
// that run the network on caller-owned device arrays.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/sphdem.h"
#include "mlp.h"
#include "mlp_tcgen05.cuh"

namespace sphdem {

static int num_sms() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return std::max(n, 1);
}

int mlp_alloc(MlpNet& m) {
    std::memset(&m, 0, sizeof(m));
    m.nparts = num_sms();
    auto al = [&](void** p, size_t b) { return cudaMalloc(p, b) == cudaSuccess; };
    bool ok = al((void**)&m.W1, sizeof(__nv_bfloat16) * MLP_H * MLP_IN) &&
              al((void**)&m.W2, sizeof(__nv_bfloat16) * MLP_H * MLP_H) &&
              al((void**)&m.W2T, sizeof(__nv_bfloat16) * MLP_H * MLP_H) &&
              al((void**)&m.b1, sizeof(float) * MLP_H) && al((void**)&m.b2, sizeof(float) * MLP_H) &&
              al((void**)&m.w3, sizeof(float) * MLP_H) && al((void**)&m.b3, sizeof(float)) &&
              al((void**)&m.master, sizeof(float) * MLP_NPARAM) && al((void**)&m.mom, sizeof(float) * MLP_NPARAM) &&
              al((void**)&m.vel, sizeof(float) * MLP_NPARAM) &&
              al((void**)&m.part, sizeof(float) * MLP_PART * (size_t)m.nparts) &&
              al((void**)&m.loss, sizeof(float) * 2) && al((void**)&m.err, sizeof(int));
    if (!ok) {
        mlp_free(m);
        return SPHDEM_E_NOMEM;
    }
    cudaMemset(m.mom, 0, sizeof(float) * MLP_NPARAM);
    cudaMemset(m.vel, 0, sizeof(float) * MLP_NPARAM);
    cudaMemset(m.err, 0, sizeof(int));
    cudaMemset(m.loss, 0, sizeof(float) * 2);
    if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, SM_TRAIN_END + SM_ALIGN) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, SM_INFER_END + SM_ALIGN) !=
            cudaSuccess)
        return SPHDEM_E_CUDA;
    return SPHDEM_OK;
}

void mlp_free(MlpNet& m) {
    void* ps[] = {m.W1, m.W2, m.W2T, m.b1, m.b2, m.w3, m.b3, m.master, m.mom, m.vel, m.part, m.loss, m.err};
    for (void* p : ps)
        if (p) cudaFree(p);
    std::memset(&m, 0, sizeof(m));
}

static MlpDev dev_view(const MlpNet& m) { return MlpDev{m.W1, m.W2, m.W2T, m.b1, m.b2, m.w3, m.b3}; }
static MlpOpt opt_view(const MlpNet& m, const double* tstep = nullptr) {
    return MlpOpt{m.master, m.mom, m.vel, m.W1, m.W2, m.W2T, m.b1, m.b2, m.w3, m.b3, m.loss, tstep};
}

// master <- params (device FP32, MLP_NPARAM), refresh the BF16 copies
int mlp_set_params(MlpNet& m, const float* params_dev, cudaStream_t st) {
    if (cudaMemcpyAsync(m.master, params_dev, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToDevice, st) !=
        cudaSuccess)
        return SPHDEM_E_CUDA;
    k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(0, m.part, opt_view(m), 0.f, 0.f, 0.f, 0.f, 1, 0);
    return cudaGetLastError() == cudaSuccess ? SPHDEM_OK : SPHDEM_E_CUDA;
}

int mlp_forward(const MlpNet& m, const void* feat, int n, float* out, cudaStream_t st, int stall) {
    if (n <= 0) return SPHDEM_OK;
    int tiles = (n + MLP_TILE - 1) / MLP_TILE;
    int grid = std::min(tiles, 2 * m.nparts);   // two CTAs per SM overlap their MMA waits
    k_mlp_infer<<<grid, 128, SM_INFER_END + SM_ALIGN, st>>>(n, (const __nv_bfloat16*)feat, dev_view(m), out, m.err,
                                                            stall);
    return cudaGetLastError() == cudaSuccess ? SPHDEM_OK : SPHDEM_E_CUDA;
}

// partial gradients of the weighted MSE into m.part (one row per CTA; rows
// of CTAs that did not run are zeroed so the sum stays over m.nparts rows)
int mlp_grad(const MlpNet& m, const void* feat, const float* target, const float* weight, int n, float inv_wsum,
             cudaStream_t st) {
    if (cudaMemsetAsync(m.part, 0, sizeof(float) * MLP_PART * (size_t)m.nparts, st) != cudaSuccess)
        return SPHDEM_E_CUDA;
    if (n <= 0) return SPHDEM_OK;
    int tiles = (n + MLP_TILE - 1) / MLP_TILE;
    int grid = std::min(tiles, m.nparts);
    k_mlp_grad<<<grid, 128, SM_TRAIN_END + SM_ALIGN, st>>>(n, (const __nv_bfloat16*)feat, target, weight, inv_wsum,
                                                            dev_view(m), m.part, m.err);
    return cudaGetLastError() == cudaSuccess ? SPHDEM_OK : SPHDEM_E_CUDA;
}

// one Adam step with the gradient in m.part (step number t from 1, or read
// from the device when tstep is given)
int mlp_adam(MlpNet& m, float lr, int t, cudaStream_t st, const double* tstep) {
    k_mlp_adam<<<(MLP_NPARAM + 2 + 255) / 256, 256, 0, st>>>(m.nparts, m.part, opt_view(m, tstep), lr, 0.9f, 0.999f,
                                                            1e-8f, t, 1);
    return cudaGetLastError() == cudaSuccess ? SPHDEM_OK : SPHDEM_E_CUDA;
}

int mlp_get_params(const MlpNet& m, float* host) {
    return cudaMemcpy(host, m.master, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost) == cudaSuccess
               ? SPHDEM_OK
               : SPHDEM_E_CUDA;
}

// He initialisation: W ~ N(0, 2/fan_in) for the hidden layers, N(0, 1/64)
// for the output, biases zero; normals from splitmix64 + Box-Muller
int mlp_init_params(MlpNet& m, unsigned seed, cudaStream_t st) {
    std::vector<float> p(MLP_NPARAM, 0.f);
    uint64_t s = 0x9E3779B97F4A7C15ull * (uint64_t)(seed + 1);
    auto next = [&]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    auto normal = [&]() { return std::sqrt(-2.0 * std::log(next())) * std::cos(6.283185307179586 * next()); };
    for (int q = 0; q < MLP_H * MLP_IN; q++) p[MLP_OFF_W1 + q] = (float)(normal() * std::sqrt(2.0 / MLP_IN));
    for (int q = 0; q < MLP_H * MLP_H; q++) p[MLP_OFF_W2 + q] = (float)(normal() * std::sqrt(2.0 / MLP_H));
    for (int q = 0; q < MLP_H; q++) p[MLP_OFF_W3 + q] = (float)(normal() * std::sqrt(1.0 / MLP_H));
    if (cudaMemcpy(m.master, p.data(), sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice) != cudaSuccess)
        return SPHDEM_E_CUDA;
    cudaMemset(m.mom, 0, sizeof(float) * MLP_NPARAM);
    cudaMemset(m.vel, 0, sizeof(float) * MLP_NPARAM);
    k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(0, m.part, opt_view(m), 0.f, 0.f, 0.f, 0.f, 1, 0);
    return cudaGetLastError() == cudaSuccess ? SPHDEM_OK : SPHDEM_E_CUDA;
}

// master <- host values, BF16 copies refreshed
int mlp_put_params(MlpNet& m, const float* host, cudaStream_t st) {
    if (cudaMemcpy(m.master, host, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice) != cudaSuccess)
        return SPHDEM_E_CUDA;
    k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(0, m.part, opt_view(m), 0.f, 0.f, 0.f, 0.f, 1, 0);
    return cudaGetLastError() == cudaSuccess ? SPHDEM_OK : SPHDEM_E_CUDA;
}

// gradient sum (MLP_NPARAM) + [sum w e^2, sum w] into out (device)
__global__ void k_mlp_sum(int nparts, const float* __restrict__ part, float* out) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < MLP_NPARAM + 2; p += gridDim.x * blockDim.x) {
        float g = 0.f;
        for (int c = 0; c < nparts; c++) g += part[(size_t)c * MLP_PART + p];
        out[p] = g;
    }
}

}  // namespace sphdem

using namespace sphdem;

// device time of the last forward / gradient kernel of this host thread
static thread_local double g_last_fwd_ms = 0.0, g_last_grad_ms = 0.0;

// CUDA events around one launch on stream st (elapsed read after the caller's sync)
struct LaunchTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    bool ok = false;
    void start(cudaStream_t st) {
        ok = cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess &&
             cudaEventRecord(a, st) == cudaSuccess;
    }
    void stop(cudaStream_t st) { ok = ok && cudaEventRecord(b, st) == cudaSuccess; }
    double ms() {
        float t = 0.f;
        if (ok && cudaEventElapsedTime(&t, a, b) != cudaSuccess) t = 0.f;
        return (double)t;
    }
    ~LaunchTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

static int mlp_oneshot(const float* params, void* stream, MlpNet& m) {
    int r = mlp_alloc(m);
    if (r) return r;
    return mlp_set_params(m, params, (cudaStream_t)stream);
}

extern "C" int sphdem_mlp_forward(const void* feat, int32_t n, const float* params, float* out, void* stream) {
    if (!feat || !params || !out || n < 0) return SPHDEM_E_ARG;
    MlpNet m;
    cudaStream_t st = (cudaStream_t)stream;
    int r = mlp_oneshot(params, stream, m);
    // failure drill of the bounded device waits (see sphdem.h)
    const char* inj = getenv("SPHDEM_FAULT_DRILL");
    int stall = (inj && strcmp(inj, "mlp_wait") == 0) ? 1 : 0;
    LaunchTimer tm;
    tm.start(st);
    if (!r) r = mlp_forward(m, feat, n, out, st, stall);
    tm.stop(st);
    int err = 0;
    if (!r && cudaMemcpyAsync(&err, m.err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) r = SPHDEM_E_CUDA;
    if (!r && cudaStreamSynchronize(st) != cudaSuccess) r = SPHDEM_E_CUDA;
    if (!r && err) r = SPHDEM_E_TIMEOUT;
    g_last_fwd_ms = r ? 0.0 : tm.ms();
    mlp_free(m);
    return r;
}

extern "C" int sphdem_mlp_grad(const void* feat, const float* target, const float* weight, int32_t n,
                               const float* params, double weight_sum, float* grad, void* stream) {
    if (!feat || !target || !weight || !params || !grad || n < 0 || !(weight_sum > 0)) return SPHDEM_E_ARG;
    MlpNet m;
    cudaStream_t st = (cudaStream_t)stream;
    int r = mlp_oneshot(params, stream, m);
    LaunchTimer tm;
    tm.start(st);
    if (!r) r = mlp_grad(m, feat, target, weight, n, (float)(1.0 / weight_sum), st);
    tm.stop(st);
    if (!r) {
        k_mlp_sum<<<(MLP_NPARAM + 2 + 255) / 256, 256, 0, st>>>(m.nparts, m.part, grad);
        if (cudaGetLastError() != cudaSuccess) r = SPHDEM_E_CUDA;
    }
    int err = 0;
    if (!r && cudaMemcpyAsync(&err, m.err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) r = SPHDEM_E_CUDA;
    if (!r && cudaStreamSynchronize(st) != cudaSuccess) r = SPHDEM_E_CUDA;
    if (!r && err) r = SPHDEM_E_TIMEOUT;
    g_last_grad_ms = r ? 0.0 : tm.ms();
    mlp_free(m);
    return r;
}

extern "C" int sphdem_mlp_last_ms(double* forward_ms, double* grad_ms) {
    if (forward_ms) *forward_ms = g_last_fwd_ms;
    if (grad_ms) *grad_ms = g_last_grad_ms;
    return SPHDEM_OK;
}

extern "C" int32_t sphdem_mlp_param_count(void) { return MLP_NPARAM; }
