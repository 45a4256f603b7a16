// mlp.h -- device buffers and host launches of the learned PPE warm start
// network (kernels in mlp_tcgen05.cuh, host side in mlp.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace sphdem {

struct MlpNet {
    __nv_bfloat16 *W1, *W2, *W2T;   // BF16 operands the MMAs read
    float *b1, *b2, *w3, *b3;
    float *master, *mom, *vel;      // FP32 parameters and Adam moments (flattened)
    float* part;                    // per-CTA partial gradients
    float* loss;                    // [sum w e^2, sum w] of the last gradient pass
    int* err;                       // bounded-wait failures of the MMA kernels
    int nparts;                     // CTAs of the gradient kernel (= SMs)
};

int mlp_alloc(MlpNet& m);
void mlp_free(MlpNet& m);
int mlp_set_params(MlpNet& m, const float* params_dev, cudaStream_t st);
int mlp_forward(const MlpNet& m, const void* feat, int n, float* out, cudaStream_t st, int stall = 0);
int mlp_grad(const MlpNet& m, const void* feat, const float* target, const float* weight, int n, float inv_wsum,
             cudaStream_t st);
int mlp_adam(MlpNet& m, float lr, int t, cudaStream_t st, const double* tstep = nullptr);
int mlp_get_params(const MlpNet& m, float* host);
int mlp_init_params(MlpNet& m, unsigned seed, cudaStream_t st);
int mlp_put_params(MlpNet& m, const float* host, cudaStream_t st);

}  // namespace sphdem
