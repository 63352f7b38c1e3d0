// Vector kernels: conversion, axpy, scaling, random states, and the
// multi-vector projection / update kernels of block classical Gram-Schmidt.
// All reductions accumulate in FP64 (products of FP32 operands are exact in
// FP64) with a compensated fixed-order combination across warps and CTAs, so
// results are reproducible run to run.
#include "rp_apply.cuh"
#include "rp_vec.cuh"

namespace rp {

int reduce_grid() { return 2 * num_sms(); }

static void *g_scratch[SCR_COUNT] = {};
static size_t g_scratch_cap[SCR_COUNT] = {};

void *scratch_get(int slot, size_t bytes, cudaStream_t st) {
    if (bytes > g_scratch_cap[slot]) {
        if (g_scratch[slot]) {
            RP_CUDA(cudaStreamSynchronize(st));
            cudaFree(g_scratch[slot]);
        }
        g_scratch[slot] = nullptr;
        g_scratch_cap[slot] = 0;
        RP_CUDA(cudaMalloc(&g_scratch[slot], bytes));
        g_scratch_cap[slot] = bytes;
    }
    return g_scratch[slot];
}

void scratch_release_all() {
    for (int s = 0; s < SCR_COUNT; s++) {
        if (g_scratch[s]) cudaFree(g_scratch[s]);
        g_scratch[s] = nullptr;
        g_scratch_cap[s] = 0;
    }
}

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

// Vectors are streamed as 16-byte packets: one complex double or two complex
// floats.  A packet count of n * sizeof(element) / 16 requires an even n for
// complex64; the element-wise kernels further down handle the odd case.
template <typename Real>
struct Packet;
template <>
struct Packet<double> {
    static constexpr int E = 1;
    double2 v;
    __device__ __forceinline__ void load(const void *p, uint64_t k) {
        v = __ldg(static_cast<const double2 *>(p) + k);
    }
    __device__ __forceinline__ void load_rw(const void *p, uint64_t k) {
        v = static_cast<const double2 *>(p)[k];
    }
    __device__ __forceinline__ double re(int) const { return v.x; }
    __device__ __forceinline__ double im(int) const { return v.y; }
    __device__ __forceinline__ void set(int, double r, double i) { v = make_double2(r, i); }
    __device__ __forceinline__ void store(void *p, uint64_t k) const {
        static_cast<double2 *>(p)[k] = v;
    }
};
template <>
struct Packet<float> {
    static constexpr int E = 2;
    float4 v;
    __device__ __forceinline__ void load(const void *p, uint64_t k) {
        v = __ldg(static_cast<const float4 *>(p) + k);
    }
    __device__ __forceinline__ void load_rw(const void *p, uint64_t k) {
        v = static_cast<const float4 *>(p)[k];
    }
    __device__ __forceinline__ double re(int e) const { return e ? v.z : v.x; }
    __device__ __forceinline__ double im(int e) const { return e ? v.w : v.y; }
    __device__ __forceinline__ void set(int e, double r, double i) {
        if (e) {
            v.z = (float)r;
            v.w = (float)i;
        } else {
            v.x = (float)r;
            v.y = (float)i;
        }
    }
    __device__ __forceinline__ void store(void *p, uint64_t k) const {
        static_cast<float4 *>(p)[k] = v;
    }
};

constexpr int DOT_G = 8;   // vectors per group of the projection kernel

// Projections <u_i | w>: each CTA owns a contiguous chunk of packets and
// takes the vectors in groups of DOT_G, reading w once per group and the
// group's vectors side by side (DOT_G + 1 independent 16-byte loads in
// flight per thread).  Per-thread FP64 sums, then a fixed-order compensated
// combination across the CTA's warps.
template <typename Real>
__global__ void __launch_bounds__(RT) k_multi_dot(uint64_t npk, const VecTable tab, int nvec,
                                                  const void *w, double *partials,
                                                  const int *gate, const int *gate2) {
    if ((gate && *gate == 0) || (gate2 && *gate2 == 0)) return;
    constexpr int E = Packet<Real>::E;
    __shared__ double scratch[RW][2 * DOT_G];
    const uint64_t chunk = (npk + gridDim.x - 1) / gridDim.x;
    const uint64_t lo = blockIdx.x * chunk;
    const uint64_t hi = lo + chunk < npk ? lo + chunk : npk;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int g0 = 0; g0 < nvec; g0 += DOT_G) {
        const int ng = nvec - g0 < DOT_G ? nvec - g0 : DOT_G;
        double sr[DOT_G], si[DOT_G];
#pragma unroll
        for (int q = 0; q < DOT_G; q++) sr[q] = si[q] = 0.0;
        for (uint64_t k = lo + threadIdx.x; k < hi; k += RT) {
            Packet<Real> wp, up[DOT_G];
            wp.load_rw(w, k);
#pragma unroll
            for (int q = 0; q < DOT_G; q++)
                if (q < ng) up[q].load(tab.p[g0 + q], k);
#pragma unroll
            for (int q = 0; q < DOT_G; q++) {
                if (q < ng) {
#pragma unroll
                    for (int e = 0; e < E; e++) {
                        const double ar = up[q].re(e), ai = up[q].im(e);
                        const double br = wp.re(e), bi = wp.im(e);
                        sr[q] = fma(ar, br, fma(ai, bi, sr[q]));
                        si[q] = fma(ar, bi, fma(-ai, br, si[q]));
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < DOT_G; q++) {
            const double a = warp_sum(sr[q]), b = warp_sum(si[q]);
            if (lane == 0) {
                scratch[warp][2 * q] = a;
                scratch[warp][2 * q + 1] = b;
            }
        }
        __syncthreads();
        if (threadIdx.x < 2 * ng) {
            CompSum c;
            for (int wi = 0; wi < RW; wi++) c.add(scratch[wi][threadIdx.x]);
            const int q = threadIdx.x >> 1;
            partials[((size_t)blockIdx.x * nvec + g0 + q) * 2 + (threadIdx.x & 1)] = c.value();
        }
        __syncthreads();
    }
}

// Element-wise fallback for a complex64 vector of odd length.
__global__ void __launch_bounds__(RT) k_multi_dot_odd(uint64_t n, const VecTable tab, int nvec,
                                                      const Cplx<float> *w, double *partials,
                                                      const int *gate, const int *gate2) {
    if ((gate && *gate == 0) || (gate2 && *gate2 == 0)) return;
    __shared__ double scratch[RW];
    const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t lo = blockIdx.x * chunk;
    const uint64_t hi = lo + chunk < n ? lo + chunk : n;
    for (int i = 0; i < nvec; i++) {
        const Cplx<float> *u = static_cast<const Cplx<float> *>(tab.p[i]);
        double sr = 0.0, si = 0.0;
        for (uint64_t k = lo + threadIdx.x; k < hi; k += RT) {
            const Cplx<float> a = u[k], b = w[k];
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
        k_multi_dot<double><<<g, RT, 0, st>>>(n, tab, nvec, w, partials, gate, gate2);
    else if (n % 2 == 0)
        k_multi_dot<float><<<g, RT, 0, st>>>(n / 2, tab, nvec, w, partials, gate, gate2);
    else
        k_multi_dot_odd<<<g, RT, 0, st>>>(n, tab, nvec, (const Cplx<float> *)w, partials, gate, gate2);
    RP_CUDA(cudaGetLastError());
}

constexpr int AXPY_G = 8;   // vectors loaded side by side by the update kernel

// w += sum_i c_i u_i and ||w||^2 in one pass: per packet of w, the vectors
// are read in groups of AXPY_G independent 16-byte loads, the update is
// accumulated in FP64 and rounded once to the vector precision.
template <typename Real>
__global__ void __launch_bounds__(RT) k_multi_axpy(uint64_t npk, const VecTable tab, int nvec,
                                                   const int *nvec_dev, const double *coef,
                                                   void *w, double *norm_partials,
                                                   const int *gate, const int *gate2) {
    if ((gate && *gate == 0) || (gate2 && *gate2 == 0)) return;
    constexpr int E = Packet<Real>::E;
    __shared__ double scratch[RW];
    __shared__ double c[2 * (MAX_KRYLOV + 1)];
    const int nv = nvec_dev ? *nvec_dev : nvec;
    for (int i = threadIdx.x; i < 2 * nv; i += RT) c[i] = coef[i];
    __syncthreads();
    const uint64_t chunk = (npk + gridDim.x - 1) / gridDim.x;
    const uint64_t lo = blockIdx.x * chunk;
    const uint64_t hi = lo + chunk < npk ? lo + chunk : npk;
    double nrm = 0.0;
    for (uint64_t k = lo + threadIdx.x; k < hi; k += RT) {
        Packet<Real> wp;
        wp.load_rw(w, k);
        double xr[E], xi[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
            xr[e] = wp.re(e);
            xi[e] = wp.im(e);
        }
        for (int i0 = 0; i0 < nv; i0 += AXPY_G) {
            Packet<Real> up[AXPY_G];
#pragma unroll
            for (int q = 0; q < AXPY_G; q++)
                if (i0 + q < nv) up[q].load(tab.p[i0 + q], k);
#pragma unroll
            for (int q = 0; q < AXPY_G; q++) {
                if (i0 + q < nv) {
                    const double cr = c[2 * (i0 + q)], ci = c[2 * (i0 + q) + 1];
#pragma unroll
                    for (int e = 0; e < E; e++) {
                        const double ur = up[q].re(e), ui = up[q].im(e);
                        xr[e] = fma(cr, ur, fma(-ci, ui, xr[e]));
                        xi[e] = fma(cr, ui, fma(ci, ur, xi[e]));
                    }
                }
            }
        }
#pragma unroll
        for (int e = 0; e < E; e++) {
            wp.set(e, xr[e], xi[e]);
            const double rr = wp.re(e), ri = wp.im(e);   // the rounded values
            nrm = fma(rr, rr, fma(ri, ri, nrm));
        }
        wp.store(w, k);
    }
    if (norm_partials) {
        const double s = block_sum(nrm, scratch);
        if (threadIdx.x == 0) norm_partials[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(RT) k_multi_axpy_odd(uint64_t n, const VecTable tab, int nvec,
                                                       const int *nvec_dev, const double *coef,
                                                       Cplx<float> *w, double *norm_partials,
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
        const Cplx<float> w0 = w[k];
        double xr = w0.x, xi = w0.y;
        for (int i = 0; i < nv; i++) {
            const Cplx<float> u = static_cast<const Cplx<float> *>(tab.p[i])[k];
            const double cr = c[2 * i], ci = c[2 * i + 1];
            xr = fma(cr, (double)u.x, fma(-ci, (double)u.y, xr));
            xi = fma(cr, (double)u.y, fma(ci, (double)u.x, xi));
        }
        const Cplx<float> r{(float)xr, (float)xi};
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
        k_multi_axpy<double><<<g, RT, 0, st>>>(n, tab, nvec, nvec_dev, coef, w, norm_partials,
                                               gate, gate2);
    else if (n % 2 == 0)
        k_multi_axpy<float><<<g, RT, 0, st>>>(n / 2, tab, nvec, nvec_dev, coef, w, norm_partials,
                                              gate, gate2);
    else
        k_multi_axpy_odd<<<g, RT, 0, st>>>(n, tab, nvec, nvec_dev, coef, (Cplx<float> *)w,
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
