// MLP of the learned Krylov step controller (host interface).
#pragma once

#include "rp_common.cuh"

namespace rp {

constexpr int MLP_HIDDEN = 64;

struct Mlp {
    int in = 0, out = 0, np = 0, step = 0;
    float *params = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
    float *io = nullptr;      // inference input/output buffer, kept between calls
    size_t io_cap = 0;        // its size in floats
};

int mlp_num_params(int in, int out);
void mlp_create(Mlp &net, int in, int out, uint64_t seed);
void mlp_free(Mlp &net);
void mlp_forward(Mlp &net, const float *X_host, int n, float *Y_host, cudaStream_t st);
// mean loss and its gradient (host copy) over n samples
float mlp_grad(Mlp &net, const float *X_host, const float *Y_host, int n, float *grad_host,
               cudaStream_t st);
// Adam over mini-batches; returns the mean loss of the last epoch
float mlp_train(Mlp &net, const float *X_host, const float *Y_host, int n, int epochs, int batch,
                float lr, uint64_t seed, cudaStream_t st);
void mlp_get(Mlp &net, float *p);
void mlp_set(Mlp &net, const float *p);

}  // namespace rp
