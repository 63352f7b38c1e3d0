// Vector kernels: conversion, axpy, scaling, random states, and the
// multi-vector projection / update kernels of block classical Gram-Schmidt.
// All reductions accumulate in FP64 (products of FP32 operands are exact in
// FP64) with a compensated fixed-order combination across warps and CTAs, so
// results are reproducible run to run.
#include "rp_apply.cuh"
#include "rp_vec.cuh"

namespace rp {

int reduce_grid() { return 2 * num_sms(); }

static inline int blocks_for(uint64_t n, int threads, int cap) {
    uint64_t b = (n + threads - 1) / threads;
    return (int)(b < (uint64_t)cap ? (b ? b : 1) : cap);
}

template <typename RO, typename RI>
__global__ void k_convert(Cplx<RO> *dst, const Cplx<RI> *src, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        Cplx<RI> v = src[i];
        dst[i] = Cplx<RO>{(RO)v.x, (RO)v.y};   // round to nearest
    }
}

void vec_convert(int dto, void *dst, int dfrom, const void *src, uint64_t n, cudaStream_t st) {
    if (!n) return;
    const int bl = blocks_for(n, 256, 8 * num_sms());
    if (dto == dfrom) {
        RP_CUDA(cudaMemcpyAsync(dst, src, n * (dto == 2 ? 16 : 8), cudaMemcpyDeviceToDevice, st));
    } else if (dto == 1) {
        k_convert<float, double><<<bl, 256, 0, st>>>((Cplx<float> *)dst, (const Cplx<double> *)src, n);
    } else {
        k_convert<double, float><<<bl, 256, 0, st>>>((Cplx<double> *)dst, (const Cplx<float> *)src, n);
    }
    RP_CUDA(cudaGetLastError());
}

template <typename Real>
__global__ void k_axpy(uint64_t n, Cplx<Real> *y, double ar, double ai, const Cplx<Real> *x) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        Cplx<Real> v = x[i], w = y[i];
        w.x = (Real)((double)w.x + ar * v.x - ai * v.y);
        w.y = (Real)((double)w.y + ar * v.y + ai * v.x);
        y[i] = w;
    }
}

void vec_axpy(int dtype, uint64_t n, void *y, double ar, double ai, const void *x,
              cudaStream_t st) {
    if (!n) return;
    const int bl = blocks_for(n, 256, 8 * num_sms());
    if (dtype == 2) k_axpy<double><<<bl, 256, 0, st>>>(n, (Cplx<double> *)y, ar, ai, (const Cplx<double> *)x);
    else k_axpy<float><<<bl, 256, 0, st>>>(n, (Cplx<float> *)y, ar, ai, (const Cplx<float> *)x);
    RP_CUDA(cudaGetLastError());
}

template <typename Real>
__global__ void k_add3(uint64_t n, Cplx<Real> *r, const Cplx<Real> *a, const Cplx<Real> *b) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        Cplx<Real> u = a[i], v = b[i];
        r[i] = Cplx<Real>{u.x + v.x, u.y + v.y};
    }
}

void vec_add3(int dtype, uint64_t n, void *res, const void *a, const void *b, cudaStream_t st) {
    if (!n) return;
    const int bl = blocks_for(n, 256, 8 * num_sms());
    if (dtype == 2) k_add3<double><<<bl, 256, 0, st>>>(n, (Cplx<double> *)res, (const Cplx<double> *)a, (const Cplx<double> *)b);
    else k_add3<float><<<bl, 256, 0, st>>>(n, (Cplx<float> *)res, (const Cplx<float> *)a, (const Cplx<float> *)b);
    RP_CUDA(cudaGetLastError());
}

template <typename Real>
__global__ void k_scale(uint64_t n, Cplx<Real> *v, double ar, double ai) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        Cplx<Real> w = v[i];
        v[i] = Cplx<Real>{(Real)(ar * w.x - ai * w.y), (Real)(ar * w.y + ai * w.x)};
    }
}

void vec_scale(int dtype, uint64_t n, void *v, double ar, double ai, cudaStream_t st) {
    if (!n) return;
    const int bl = blocks_for(n, 256, 8 * num_sms());
    if (dtype == 2) k_scale<double><<<bl, 256, 0, st>>>(n, (Cplx<double> *)v, ar, ai);
    else k_scale<float><<<bl, 256, 0, st>>>(n, (Cplx<float> *)v, ar, ai);
    RP_CUDA(cudaGetLastError());
}

// Counter-based normal deviates: splitmix64 hash of (seed, index) -> two
// uniforms -> Box-Muller.  Deterministic for a given seed.
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

template <typename Real>
__global__ void k_random(uint64_t n, Cplx<Real> *v, uint64_t seed) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t h1 = splitmix64(seed * 0x632BE59BD9B4E019ull + 2 * i);
        uint64_t h2 = splitmix64(seed * 0x632BE59BD9B4E019ull + 2 * i + 1);
        double u1 = ((h1 >> 11) + 1) * (1.0 / 9007199254740993.0);   // (0, 1]
        double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);         // [0, 1)
        double r = sqrt(-2.0 * log(u1));
        double s, c;
        sincospi(2.0 * u2, &s, &c);
        v[i] = Cplx<Real>{(Real)(r * c), (Real)(r * s)};
    }
}

void vec_random(int dtype, uint64_t n, void *v, uint64_t seed, cudaStream_t st) {
    if (!n) return;
    const int bl = blocks_for(n, 256, 8 * num_sms());
    if (dtype == 2) k_random<double><<<bl, 256, 0, st>>>(n, (Cplx<double> *)v, seed);
    else k_random<float><<<bl, 256, 0, st>>>(n, (Cplx<float> *)v, seed);
    RP_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Block Gram-Schmidt kernels
// ---------------------------------------------------------------------------
constexpr int RT = 256;   // threads of the reduction kernels
constexpr int RW = RT / 32;

// Block-level fixed-order compensated sum of one double per thread;
// result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *scratch) {
    v = warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
        CompSum c;
        for (int w = 0; w < RW; w++) c.add(scratch[w]);
        r = c.value();
    }
    return r;
}

// Each CTA owns a contiguous chunk of elements.  For every vector u_i it sums
// conj(u_i) * w over the chunk; w is re-read from L2/L1 per vector.
template <typename Real>
__global__ void __launch_bounds__(RT) k_multi_dot(uint64_t n, const VecTable tab, int nvec,
                                                  const Cplx<Real> *w, double *partials,
                                                  const int *gate, const int *gate2) {
    if ((gate && *gate == 0) || (gate2 && *gate2 == 0)) return;
    __shared__ double scratch[RW];
    const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t lo = blockIdx.x * chunk;
    const uint64_t hi = lo + chunk < n ? lo + chunk : n;
    for (int i = 0; i < nvec; i++) {
        const Cplx<Real> *u = static_cast<const Cplx<Real> *>(tab.p[i]);
        double sr = 0.0, si = 0.0;
        for (uint64_t k = lo + threadIdx.x; k < hi; k += RT) {
            const Cplx<Real> a = u[k], b = w[k];
            sr = fma((double)a.x, (double)b.x, fma((double)a.y, (double)b.y, sr));
            si = fma((double)a.x, (double)b.y, fma(-(double)a.y, (double)b.x, si));
        }
        const double r0 = block_sum(sr, scratch);
        const double r1 = block_sum(si, scratch);
        if (threadIdx.x == 0) {
            partials[((size_t)blockIdx.x * nvec + i) * 2 + 0] = r0;
            partials[((size_t)blockIdx.x * nvec + i) * 2 + 1] = r1;
        }
    }
}

void multi_dot_partials(int dtype, uint64_t n, const VecTable &tab, int nvec, const void *w,
                        double *partials, const int *gate, const int *gate2, cudaStream_t st) {
    RP_REQUIRE(nvec >= 0 && nvec <= MAX_KRYLOV + 1, -2, "too many vectors");
    const int g = reduce_grid();
    if (dtype == 2)
        k_multi_dot<double><<<g, RT, 0, st>>>(n, tab, nvec, (const Cplx<double> *)w, partials, gate, gate2);
    else
        k_multi_dot<float><<<g, RT, 0, st>>>(n, tab, nvec, (const Cplx<float> *)w, partials, gate, gate2);
    RP_CUDA(cudaGetLastError());
}

template <typename Real>
__global__ void __launch_bounds__(RT) k_multi_axpy(uint64_t n, const VecTable tab, int nvec,
                                                   const int *nvec_dev, const double *coef,
                                                   Cplx<Real> *w, double *norm_partials,
                                                   const int *gate, const int *gate2) {
    if ((gate && *gate == 0) || (gate2 && *gate2 == 0)) return;
    __shared__ double scratch[RW];
    __shared__ double c[2 * (MAX_KRYLOV + 1)];
    const int nv = nvec_dev ? *nvec_dev : nvec;
    for (int i = threadIdx.x; i < 2 * nv; i += RT) c[i] = coef[i];
    __syncthreads();
    const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t lo = blockIdx.x * chunk;
    const uint64_t hi = lo + chunk < n ? lo + chunk : n;
    double nrm = 0.0;
    for (uint64_t k = lo + threadIdx.x; k < hi; k += RT) {
        const Cplx<Real> w0 = w[k];
        double xr = w0.x, xi = w0.y;
        for (int i = 0; i < nv; i++) {
            const Cplx<Real> u = static_cast<const Cplx<Real> *>(tab.p[i])[k];
            const double cr = c[2 * i], ci = c[2 * i + 1];
            xr = fma(cr, (double)u.x, fma(-ci, (double)u.y, xr));
            xi = fma(cr, (double)u.y, fma(ci, (double)u.x, xi));
        }
        const Cplx<Real> r{(Real)xr, (Real)xi};
        w[k] = r;
        nrm = fma((double)r.x, (double)r.x, fma((double)r.y, (double)r.y, nrm));
    }
    if (norm_partials) {
        const double s = block_sum(nrm, scratch);
        if (threadIdx.x == 0) norm_partials[blockIdx.x] = s;
    }
}

void multi_axpy(int dtype, uint64_t n, const VecTable &tab, int nvec, const int *nvec_dev,
                const double *coef, void *w, double *norm_partials, const int *gate,
                const int *gate2, cudaStream_t st) {
    RP_REQUIRE(nvec >= 0 && nvec <= MAX_KRYLOV + 1, -2, "too many vectors");
    const int g = reduce_grid();
    if (dtype == 2)
        k_multi_axpy<double><<<g, RT, 0, st>>>(n, tab, nvec, nvec_dev, coef, (Cplx<double> *)w,
                                               norm_partials, gate, gate2);
    else
        k_multi_axpy<float><<<g, RT, 0, st>>>(n, tab, nvec, nvec_dev, coef, (Cplx<float> *)w,
                                              norm_partials, gate, gate2);
    RP_CUDA(cudaGetLastError());
}

__global__ void k_reduce_partials(const double *partials, int grid, int n, double *out) {
    for (int i = threadIdx.x; i < 2 * n; i += blockDim.x) {
        CompSum c;
        for (int g = 0; g < grid; g++) c.add(partials[(size_t)g * 2 * n + i]);
        out[i] = c.value();
    }
}

void reduce_partials(const double *partials, int grid, int n, double *out, cudaStream_t st) {
    k_reduce_partials<<<1, 128, 0, st>>>(partials, grid, n, out);
    RP_CUDA(cudaGetLastError());
}

}  // namespace rp
