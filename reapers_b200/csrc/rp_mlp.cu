// Small MLP (in -> 64 -> 64 -> out, tanh hidden layers, linear output) for
// the learned Krylov step controller: hand-written CUDA forward, backward and
// Adam kernels, FP32.  Parameters are one flat array
// [W1 (64 x in), b1, W2 (64 x 64), b2, W3 (out x 64), b3], row-major.
//
// Training step on a mini-batch: k_mlp_grad runs one CTA of 64 threads per
// slice of samples (thread j = hidden unit j), keeps the weights and its
// gradient partial in shared memory, and writes the partial to global memory;
// k_mlp_reduce sums the partials in a fixed order (reproducible) and
// k_mlp_adam applies Adam.  Loss: mean squared error / 2.
#include <cmath>
#include <vector>

#include "rp_common.cuh"
#include "rp_mlp.cuh"

namespace rp {

constexpr int HID = MLP_HIDDEN;

int mlp_num_params(int in, int out) { return HID * in + HID + HID * HID + HID + out * HID + out; }

struct MlpDims {
    int in, out, np;
    int oW1, ob1, oW2, ob2, oW3, ob3;
};

static MlpDims dims(int in, int out) {
    MlpDims d;
    d.in = in;
    d.out = out;
    d.oW1 = 0;
    d.ob1 = d.oW1 + HID * in;
    d.oW2 = d.ob1 + HID;
    d.ob2 = d.oW2 + HID * HID;
    d.oW3 = d.ob2 + HID;
    d.ob3 = d.oW3 + out * HID;
    d.np = d.ob3 + out;
    return d;
}

// forward for one sample held in shared memory; thread j = hidden unit j
__device__ __forceinline__ void fwd_sample(const MlpDims &d, const float *P, const float *x,
                                           float *h1, float *h2, float *y) {
    const int j = threadIdx.x;
    float a = P[d.ob1 + j];
    for (int i = 0; i < d.in; i++) a = fmaf(P[d.oW1 + j * d.in + i], x[i], a);
    h1[j] = tanhf(a);
    __syncthreads();
    float b = P[d.ob2 + j];
    for (int k = 0; k < HID; k++) b = fmaf(P[d.oW2 + j * HID + k], h1[k], b);
    h2[j] = tanhf(b);
    __syncthreads();
    if (j < d.out) {
        float c = P[d.ob3 + j];
        for (int k = 0; k < HID; k++) c = fmaf(P[d.oW3 + j * HID + k], h2[k], c);
        y[j] = c;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(HID) k_mlp_forward(MlpDims d, const float *params, const float *X,
                                                     int n, float *Y) {
    extern __shared__ float sm[];
    float *P = sm, *x = P + d.np, *h1 = x + d.in, *h2 = h1 + HID, *y = h2 + HID;
    for (int i = threadIdx.x; i < d.np; i += HID) P[i] = params[i];
    __syncthreads();
    for (int s = blockIdx.x; s < n; s += gridDim.x) {
        for (int i = threadIdx.x; i < d.in; i += HID) x[i] = X[(size_t)s * d.in + i];
        __syncthreads();
        fwd_sample(d, P, x, h1, h2, y);
        if (threadIdx.x < d.out) Y[(size_t)s * d.out + threadIdx.x] = y[threadIdx.x];
        __syncthreads();
    }
}

// Gradient partial of one CTA over samples [s0, s1) of the batch.
__global__ void __launch_bounds__(HID) k_mlp_grad(MlpDims d, const float *params, const float *X,
                                                  const float *Y, int n, int per_cta, float *gpart,
                                                  float *lpart) {
    extern __shared__ float sm[];
    float *P = sm, *G = P + d.np, *x = G + d.np, *h1 = x + d.in, *h2 = h1 + HID, *y = h2 + HID;
    float *dy = y + 8, *dh2 = dy + 8, *dh1 = dh2 + HID;
    const int j = threadIdx.x;
    for (int i = j; i < d.np; i += HID) {
        P[i] = params[i];
        G[i] = 0.f;
    }
    __syncthreads();
    float loss = 0.f;
    const int s0 = blockIdx.x * per_cta, s1 = min(n, s0 + per_cta);
    for (int s = s0; s < s1; s++) {
        for (int i = j; i < d.in; i += HID) x[i] = X[(size_t)s * d.in + i];
        __syncthreads();
        fwd_sample(d, P, x, h1, h2, y);
        if (j < d.out) {
            const float e = y[j] - Y[(size_t)s * d.out + j];
            dy[j] = e;
            loss += 0.5f * e * e;
        }
        __syncthreads();
        // output layer
        for (int o = 0; o < d.out; o++) G[d.oW3 + o * HID + j] += dy[o] * h2[j];
        if (j < d.out) G[d.ob3 + j] += dy[j];
        float g2 = 0.f;
        for (int o = 0; o < d.out; o++) g2 = fmaf(P[d.oW3 + o * HID + j], dy[o], g2);
        dh2[j] = g2 * (1.f - h2[j] * h2[j]);
        __syncthreads();
        // second hidden layer: thread j owns row j of W2
        for (int k = 0; k < HID; k++) G[d.oW2 + j * HID + k] += dh2[j] * h1[k];
        G[d.ob2 + j] += dh2[j];
        float g1 = 0.f;
        for (int k = 0; k < HID; k++) g1 = fmaf(P[d.oW2 + k * HID + j], dh2[k], g1);
        dh1[j] = g1 * (1.f - h1[j] * h1[j]);
        __syncthreads();
        for (int i = 0; i < d.in; i++) G[d.oW1 + j * d.in + i] += dh1[j] * x[i];
        G[d.ob1 + j] += dh1[j];
        __syncthreads();
    }
    for (int i = j; i < d.np; i += HID) gpart[(size_t)blockIdx.x * d.np + i] = G[i];
    // loss of this CTA (thread order fixed)
    __shared__ float ls[HID];
    ls[j] = loss;
    __syncthreads();
    if (j == 0) {
        float t = 0.f;
        for (int k = 0; k < HID; k++) t += ls[k];
        lpart[blockIdx.x] = t;
    }
}

// g = scale * sum of the per-CTA partials: a block of 32 parameters x 8
// warps, warp y taking partials y, y + 8, ..., then the 8 sums in order.
__global__ void __launch_bounds__(256) k_mlp_reduce(int np, int nparts, const float *gpart,
                                                    float scale, float *g) {
    __shared__ double red[8][33];
    const int x = threadIdx.x & 31, y = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + x;
    double sum = 0.0;
    if (i < np)
        for (int p = y; p < nparts; p += 8) sum += gpart[(size_t)p * np + i];
    red[y][x] = sum;
    __syncthreads();
    if (y == 0 && i < np) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += red[w][x];
        g[i] = (float)(t * scale);
    }
}

__global__ void k_mlp_adam(int np, float *params, const float *g, float *m, float *v, float lr,
                           float b1, float b2, float eps, int step) {
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// ---------------------------------------------------------------------------
// Host
// ---------------------------------------------------------------------------
static size_t fwd_smem(const MlpDims &d) {
    return (size_t)(d.np + d.in + 2 * HID + 8) * sizeof(float);
}
static size_t grad_smem(const MlpDims &d) {
    return (size_t)(2 * d.np + d.in + 4 * HID + 16) * sizeof(float);
}

void mlp_create(Mlp &net, int in, int out, uint64_t seed) {
    RP_REQUIRE(in >= 1 && in <= 256 && out >= 1 && out <= 8, -2, "MLP dims: in 1..256, out 1..8");
    net.in = in;
    net.out = out;
    net.np = mlp_num_params(in, out);
    std::vector<float> p(net.np, 0.f);
    // Glorot-uniform weights from a splitmix64 stream, zero biases
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
    auto rnd = [&]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) / 9007199254740992.0;
    };
    const MlpDims d = dims(in, out);
    auto fill = [&](int off, int rows, int cols) {
        const double a = std::sqrt(6.0 / (rows + cols));
        for (int k = 0; k < rows * cols; k++) p[off + k] = (float)((2 * rnd() - 1) * a);
    };
    fill(d.oW1, HID, in);
    fill(d.oW2, HID, HID);
    fill(d.oW3, out, HID);
    RP_CUDA(cudaMalloc((void **)&net.params, net.np * sizeof(float)));
    RP_CUDA(cudaMalloc((void **)&net.m, net.np * sizeof(float)));
    RP_CUDA(cudaMalloc((void **)&net.v, net.np * sizeof(float)));
    RP_CUDA(cudaMalloc((void **)&net.g, net.np * sizeof(float)));
    RP_CUDA(cudaMemcpy(net.params, p.data(), net.np * sizeof(float), cudaMemcpyHostToDevice));
    RP_CUDA(cudaMemset(net.m, 0, net.np * sizeof(float)));
    RP_CUDA(cudaMemset(net.v, 0, net.np * sizeof(float)));
    net.step = 0;
    RP_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)grad_smem(d)));
    RP_CUDA(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fwd_smem(d)));
}

void mlp_free(Mlp &net) {
    if (net.params) cudaFree(net.params);
    if (net.m) cudaFree(net.m);
    if (net.v) cudaFree(net.v);
    if (net.g) cudaFree(net.g);
    if (net.io) cudaFree(net.io);
    net = Mlp{};
}

void mlp_forward(Mlp &net, const float *X_host, int n, float *Y_host, cudaStream_t st) {
    const MlpDims d = dims(net.in, net.out);
    const size_t need = (size_t)n * (d.in + d.out);
    if (need > net.io_cap) {
        RP_CUDA(cudaStreamSynchronize(st));
        if (net.io) cudaFree(net.io);
        net.io = nullptr;
        net.io_cap = 0;
        RP_CUDA(cudaMalloc((void **)&net.io, need * sizeof(float)));
        net.io_cap = need;
    }
    float *dX = net.io, *dY = net.io + (size_t)n * d.in;
    RP_CUDA(cudaMemcpyAsync(dX, X_host, (size_t)n * d.in * sizeof(float), cudaMemcpyHostToDevice, st));
    const int grid = std::min(std::max(n, 1), 4 * 148);
    k_mlp_forward<<<grid, HID, fwd_smem(d), st>>>(d, net.params, dX, n, dY);
    RP_CUDA(cudaGetLastError());
    RP_CUDA(cudaMemcpyAsync(Y_host, dY, (size_t)n * d.out * sizeof(float), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
}

// gradient of the mean loss over samples [0, n) of device arrays; returns loss
static float grad_device(Mlp &net, const float *dX, const float *dY, int n, float *gpart,
                         float *lpart, cudaStream_t st) {
    const MlpDims d = dims(net.in, net.out);
    const int per = std::max(1, (n + 2 * 148 - 1) / (2 * 148));
    const int nparts = (n + per - 1) / per;
    k_mlp_grad<<<nparts, HID, grad_smem(d), st>>>(d, net.params, dX, dY, n, per, gpart, lpart);
    RP_CUDA(cudaGetLastError());
    k_mlp_reduce<<<(d.np + 31) / 32, 256, 0, st>>>(d.np, nparts, gpart, 1.f / n, net.g);
    RP_CUDA(cudaGetLastError());
    std::vector<float> lp(nparts);
    RP_CUDA(cudaMemcpyAsync(lp.data(), lpart, nparts * sizeof(float), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
    double l = 0.0;
    for (float v : lp) l += v;
    return (float)(l / n);
}

float mlp_grad(Mlp &net, const float *X_host, const float *Y_host, int n, float *grad_host,
               cudaStream_t st) {
    const MlpDims d = dims(net.in, net.out);
    RP_REQUIRE(n >= 1, -2, "no samples");
    float *dX, *dY, *gp, *lp;
    const int nparts = std::min(n, 2 * 148);
    RP_CUDA(cudaMalloc((void **)&dX, (size_t)n * d.in * sizeof(float)));
    RP_CUDA(cudaMalloc((void **)&dY, (size_t)n * d.out * sizeof(float)));
    RP_CUDA(cudaMalloc((void **)&gp, (size_t)(nparts + 1) * d.np * sizeof(float)));
    RP_CUDA(cudaMalloc((void **)&lp, (size_t)(nparts + 1) * sizeof(float)));
    RP_CUDA(cudaMemcpyAsync(dX, X_host, (size_t)n * d.in * sizeof(float), cudaMemcpyHostToDevice, st));
    RP_CUDA(cudaMemcpyAsync(dY, Y_host, (size_t)n * d.out * sizeof(float), cudaMemcpyHostToDevice, st));
    const float loss = grad_device(net, dX, dY, n, gp, lp, st);
    RP_CUDA(cudaMemcpy(grad_host, net.g, d.np * sizeof(float), cudaMemcpyDeviceToHost));
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(gp);
    cudaFree(lp);
    return loss;
}

float mlp_train(Mlp &net, const float *X_host, const float *Y_host, int n, int epochs, int batch,
                float lr, uint64_t seed, cudaStream_t st) {
    const MlpDims d = dims(net.in, net.out);
    RP_REQUIRE(n >= 1 && epochs >= 1 && batch >= 1, -2, "bad training arguments");
    // shuffle once per epoch on the host (deterministic), upload epoch order
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    std::vector<float> Xs((size_t)n * d.in), Ys((size_t)n * d.out);
    float *dX, *dY, *gp, *lp;
    const int nparts = std::min(batch, 2 * 148);
    RP_CUDA(cudaMalloc((void **)&dX, (size_t)n * d.in * sizeof(float)));
    RP_CUDA(cudaMalloc((void **)&dY, (size_t)n * d.out * sizeof(float)));
    RP_CUDA(cudaMalloc((void **)&gp, (size_t)(nparts + 1) * d.np * sizeof(float)));
    RP_CUDA(cudaMalloc((void **)&lp, (size_t)(nparts + 1) * sizeof(float)));
    uint64_t s = seed * 6364136223846793005ull + 1442695040888963407ull;
    float last = 0.f;
    for (int e = 0; e < epochs; e++) {
        for (int i = n - 1; i > 0; i--) {
            s = s * 6364136223846793005ull + 1442695040888963407ull;
            const int k = (int)((s >> 33) % (uint64_t)(i + 1));
            std::swap(idx[i], idx[k]);
        }
        for (int i = 0; i < n; i++) {
            std::copy(X_host + (size_t)idx[i] * d.in, X_host + (size_t)(idx[i] + 1) * d.in,
                      Xs.begin() + (size_t)i * d.in);
            std::copy(Y_host + (size_t)idx[i] * d.out, Y_host + (size_t)(idx[i] + 1) * d.out,
                      Ys.begin() + (size_t)i * d.out);
        }
        RP_CUDA(cudaMemcpyAsync(dX, Xs.data(), Xs.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        RP_CUDA(cudaMemcpyAsync(dY, Ys.data(), Ys.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        double tot = 0.0;
        int nb = 0;
        for (int b0 = 0; b0 < n; b0 += batch) {
            const int nb_s = std::min(batch, n - b0);
            tot += grad_device(net, dX + (size_t)b0 * d.in, dY + (size_t)b0 * d.out, nb_s, gp, lp, st);
            nb++;
            net.step++;
            k_mlp_adam<<<(d.np + 255) / 256, 256, 0, st>>>(d.np, net.params, net.g, net.m, net.v, lr,
                                                           0.9f, 0.999f, 1e-8f, net.step);
            RP_CUDA(cudaGetLastError());
        }
        last = (float)(tot / nb);
    }
    RP_CUDA(cudaStreamSynchronize(st));
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(gp);
    cudaFree(lp);
    return last;
}

void mlp_get(Mlp &net, float *p) {
    RP_CUDA(cudaMemcpy(p, net.params, net.np * sizeof(float), cudaMemcpyDeviceToHost));
}
void mlp_set(Mlp &net, const float *p) {
    RP_CUDA(cudaMemcpy(net.params, p, net.np * sizeof(float), cudaMemcpyHostToDevice));
    RP_CUDA(cudaMemset(net.m, 0, net.np * sizeof(float)));
    RP_CUDA(cudaMemset(net.v, 0, net.np * sizeof(float)));
    net.step = 0;
}

}  // namespace rp
