// Batched OTOC on one GPU: one persistent launch per time step.
//
// Work item = one problem (a disorder realisation x random state, any qubit
// count).  A CTA takes items from an atomic queue and runs the whole OTOC
// point for its item alone, in the operator order of
// examples/simple-syk-krylov.cc:42-57 at beta = 0:
//     psi = V psi0; e^{-iHt}; W; e^{iHt}; V; e^{-iHt}; W; e^{iHt}; <psi0|psi>,
// each evolve being the reference's restarted Krylov (inc/algo.h:77-173,
// 267-365: same pass criterion, breakdown rule, Hfull growth and ||Hexp0||
// test) executed by the CTA: H.psi through a 4-stage bulk-copy ring of
// 2^B-element source tiles in shared memory (tile exponent B per problem,
// chosen by the autotuner), projections and updates as CTA-wide passes with
// FP64 accumulation, FP64 H / Hfull / Pade-13 exponential in per-CTA global
// scratch.  Problems are independent, so CTAs never wait on one another.
// Vectors are FP32 (the mixed-precision form); everything else FP64.
#include <algorithm>
#include <cstring>

#include "rp_batch.cuh"
#include "rp_expm_impl.cuh"

namespace rp {

constexpr int BT = 256;          // threads per CTA
constexpr int BNW = BT / 32;
constexpr int BST = 4;           // shared-memory stages of the H.psi ring
constexpr int BMAXK = 32;        // largest krydim of the batched form

struct BatchArgs {
    const BatchProblem *probs;
    int nprob, krydim, max_restarts, ti, ntimes, hcap;
    int probe;          // > 0: only `probe` H.psi products per item (tuning)
    double t, tol;
    double *F;
    int *applies;
    char *ws;
    size_t ws_stride, vec_stride;
    int *counter;
    unsigned *err;
};

struct BatchShared {
    double red[2 * BNW];
    double sigma[BMAXK + 1];
    double hacc[2 * (BMAXK + 1)];
    double coef[2 * (BMAXK + 1)];
    double nrm;
    Cplx<float> *u[BMAXK + 1];
    int item;
};

__device__ __forceinline__ void proxy_fence_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Fixed-order sums over the CTA, broadcast to every thread.
__device__ __forceinline__ void cta_sum2(double &a, double &b, double *red) {
    a = warp_sum(a);
    b = warp_sum(b);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = a;
        red[BNW + (threadIdx.x >> 5)] = b;
    }
    __syncthreads();
    CompSum ca, cb;
    for (int w = 0; w < BNW; w++) {
        ca.add(red[w]);
        cb.add(red[BNW + w]);
    }
    a = ca.value();
    b = cb.value();
}

// <a|b> over n elements.
__device__ void cta_dot(const Cplx<float> *a, const Cplx<float> *b, uint32_t n, double *red,
                        double &re, double &im) {
    double sr = 0.0, si = 0.0;
    for (uint32_t k = threadIdx.x; k < n; k += BT) {
        const Cplx<float> x = a[k], y = b[k];
        sr = fma((double)x.x, (double)y.x, fma((double)x.y, (double)y.y, sr));
        si = fma((double)x.x, (double)y.y, fma(-(double)x.y, (double)y.x, si));
    }
    cta_sum2(sr, si, red);
    re = sr;
    im = si;
}

__device__ void cta_copy(Cplx<float> *dst, const Cplx<float> *src, uint32_t n) {
    for (uint32_t k = threadIdx.x; k < n; k += BT) dst[k] = src[k];
    proxy_fence_global();
    __syncthreads();
}

__device__ void cta_zero(Cplx<float> *dst, uint32_t n) {
    for (uint32_t k = threadIdx.x; k < n; k += BT) dst[k] = Cplx<float>{0.f, 0.f};
    proxy_fence_global();
    __syncthreads();
}

// out[k] = c (-1)^popc(z & (k ^ x)) in[k ^ x]  (SpinOp::apply, inc/ops.h:421-440)
__device__ void cta_string(uint32_t x, uint32_t z, float cr, float ci, const Cplx<float> *in,
                           Cplx<float> *out, uint32_t n) {
    for (uint32_t k = threadIdx.x; k < n; k += BT) {
        const uint32_t m = k ^ x;
        const float s = (__popc(z & m) & 1) ? -1.f : 1.f;
        const Cplx<float> v = in[m];
        out[k] = Cplx<float>{s * (cr * v.x - ci * v.y), s * (cr * v.y + ci * v.x)};
    }
    proxy_fence_global();
    __syncthreads();
}

// w += sum_{i < nv} coef_i u_i, returning ||w||^2 when want_norm.
__device__ double cta_axpy(Cplx<float> *const *u, const double *coef, int nv, Cplx<float> *w,
                           uint32_t n, double *red, bool want_norm) {
    double nrm = 0.0;
    for (uint32_t k = threadIdx.x; k < n; k += BT) {
        const Cplx<float> w0 = w[k];
        double xr = w0.x, xi = w0.y;
        for (int i = 0; i < nv; i++) {
            const Cplx<float> v = u[i][k];
            const double cr = coef[2 * i], ci = coef[2 * i + 1];
            xr = fma(cr, (double)v.x, fma(-ci, (double)v.y, xr));
            xi = fma(cr, (double)v.y, fma(ci, (double)v.x, xi));
        }
        const Cplx<float> r{(float)xr, (float)xi};
        w[k] = r;
        nrm = fma((double)r.x, (double)r.x, fma((double)r.y, (double)r.y, nrm));
    }
    proxy_fence_global();
    double dummy = 0.0;
    if (want_norm) {
        cta_sum2(nrm, dummy, red);
    } else {
        __syncthreads();
    }
    return nrm;
}

// out = scale * H in, source tiles streamed through the shared-memory ring.
// git counts ring items across calls (stage = git % BST, parity (git/BST)&1).
template <int B>
__device__ bool cta_apply(const BatchProblem &P, const Cplx<float> *in, Cplx<float> *out,
                          double scale, unsigned char *stages, uint64_t *full, long &git,
                          unsigned *err) {
    constexpr int TILE = 1 << B, E = TILE / BT;
    constexpr unsigned TB = TILE * sizeof(Cplx<float>);
    const long total = (long)P.ntiles * P.ngroups;
    const uint32_t t = threadIdx.x;
    auto issue = [&](long i) {
        const long gi = git + i;
        const int s = (int)(gi % BST);
        const int o = (int)(i / P.ngroups), g = (int)(i % P.ngroups);
        const uint32_t src = (uint32_t)o ^ P.groups[g].xh;
        mbar_arrive_expect_tx(&full[s], TB);
        bulk_g2s(stages + (size_t)s * TB, in + ((size_t)src << B), TB, &full[s]);
    };
    if (t == 0) {
        proxy_fence_global();
        for (long i = 0; i < BST - 1 && i < total; i++) issue(i);
    }
    float ar[E], ai[E];
    for (long it = 0; it < total; ++it) {
        const long gi = git + it;
        const int s = (int)(gi % BST);
        const unsigned par = (unsigned)((gi / BST) & 1);
        const int o = (int)(it / P.ngroups), g = (int)(it % P.ngroups);
        const bool okw = mbar_wait_bounded(&full[s], par, err);
        if (!__syncthreads_and(okw)) {
            // drain the copies still in flight, then give up
            if (t == 0)
                for (long i = it; i < it + BST - 1 && i < total; i++)
                    mbar_wait_bounded(&full[(git + i) % BST], (unsigned)(((git + i) / BST) & 1), err);
            __syncthreads();
            git += total;
            return false;
        }
        // every thread is past this item's barrier, so the stage of item it-1
        // is free: prefetch item it + BST - 1 into it
        if (t == 0 && it + BST - 1 < total) issue(it + BST - 1);
        if (g == 0) {
#pragma unroll
            for (int j = 0; j < E; j++) ar[j] = ai[j] = 0.f;
        }
        const Cplx<float> *tile = reinterpret_cast<const Cplx<float> *>(stages + (size_t)s * TB);
        const GroupDesc gd = P.groups[g];
        const uint32_t src_hi = ((uint32_t)o ^ gd.xh) << B;
        for (uint32_t k = gd.first; k < gd.first + gd.count; ++k) {
            const uint4 td = __ldg(reinterpret_cast<const uint4 *>(&P.terms[k]));
            const float cr = __ldg(&P.terms[k].cr), ci = __ldg(&P.terms[k].ci);
            const uint32_t xl = td.x, z = td.y, js = td.z, kind = td.w;
            const uint32_t a0 = t ^ xl;
            const uint32_t m0 = src_hi | (a0 & (uint32_t)(BT - 1));
            const uint32_t s0 = (uint32_t)(__popc(z & m0) & 1) << 31;
#pragma unroll
            for (int j = 0; j < E; j++) {
                const Cplx<float> v = tile[a0 ^ (uint32_t)(j * BT)];
                const uint32_t sb = s0 ^ ((js << (31 - j)) & 0x80000000u);
                if (kind == COEFF_REAL) {
                    const float c = __uint_as_float(__float_as_uint(cr) ^ sb);
                    ar[j] = fmaf(c, v.x, ar[j]);
                    ai[j] = fmaf(c, v.y, ai[j]);
                } else if (kind == COEFF_IMAG) {
                    const float c = __uint_as_float(__float_as_uint(ci) ^ sb);
                    ar[j] = fmaf(-c, v.y, ar[j]);
                    ai[j] = fmaf(c, v.x, ai[j]);
                } else {
                    const float c1 = __uint_as_float(__float_as_uint(cr) ^ sb);
                    const float c2 = __uint_as_float(__float_as_uint(ci) ^ sb);
                    ar[j] = fmaf(c1, v.x, fmaf(-c2, v.y, ar[j]));
                    ai[j] = fmaf(c1, v.y, fmaf(c2, v.x, ai[j]));
                }
            }
        }
        if (g == P.ngroups - 1) {
            Cplx<float> *op = out + ((size_t)o << B) + t;
#pragma unroll
            for (int j = 0; j < E; j++)
                op[(size_t)j * BT] = Cplx<float>{(float)(scale * ar[j]), (float)(scale * ai[j])};
        }
    }
    git += total;
    proxy_fence_global();
    __syncthreads();
    return true;
}

// psi <- exp(-i t H) psi by the reference's restarted Krylov, run by one CTA.
template <int B>
__device__ bool cta_evolve(const BatchProblem &P, Cplx<float> *psi, double t_real,
                           const BatchArgs &a, char *slot, BatchShared &S, unsigned char *stages,
                           uint64_t *full, double *esmem, long &git, int &applies) {
    if (t_real == 0.0) return true;   // State::evolve returns at t = beta = 0
    const uint32_t n = 1u << P.len;
    const int m = a.krydim;
    const double eta = 1.0 / sqrt(2.0);
    Cplx<float> *y = reinterpret_cast<Cplx<float> *>(slot + (size_t)(m + 1) * a.vec_stride);
    cd *H = reinterpret_cast<cd *>(slot + (size_t)(m + 4) * a.vec_stride);
    cd *hfull = H + m * m;
    cd *escr = hfull + (size_t)a.hcap * a.hcap;
    if (threadIdx.x == 0)
        for (int i = 0; i <= m; i++)
            S.u[i] = reinterpret_cast<Cplx<float> *>(slot + (size_t)i * a.vec_stride);
    __syncthreads();
    double b2, dummy;
    cta_dot(psi, psi, n, S.red, b2, dummy);
    const double beta0 = sqrt(b2);
    if (beta0 == 0.0) return true;
    cta_copy(S.u[0], psi, n);
    cta_zero(y, n);
    if (threadIdx.x == 0) S.sigma[0] = 1.0 / beta0;
    __syncthreads();
    double oldbeta = 0.0, beta = 0.0;
    for (int cycle = 1;; cycle++) {
        const int base = (cycle - 1) * m;
        if (base + m > a.hcap) {   // bounded by max_restarts on the host; defensive
            atomicOr(a.err, DEV_ERR_BOUNDS);
            return false;
        }
        for (int e = threadIdx.x; e < 2 * m * m; e += BT) reinterpret_cast<double *>(H)[e] = 0.0;
        __syncthreads();
        int m_eff = m;
        bool brokedown = false;
        for (int j = 0; j < m; j++) {
            Cplx<float> *w = S.u[j + 1];
            if (!cta_apply<B>(P, S.u[j], w, S.sigma[j], stages, full, git, a.err)) return false;
            applies++;
            double old = 1.0, norm = eta / 2;
            int niter = 0;
            while (niter < 3 && norm != 0.0 && norm < eta * old) {
                niter++;
                for (int i = 0; i <= j; i++) {
                    double hr, hi;
                    cta_dot(S.u[i], w, n, S.red, hr, hi);
                    const double sg = S.sigma[i];
                    hr *= sg;
                    hi *= sg;
                    if (threadIdx.x == 0) {
                        S.hacc[2 * i] = (niter == 1 ? 0.0 : S.hacc[2 * i]) + hr;
                        S.hacc[2 * i + 1] = (niter == 1 ? 0.0 : S.hacc[2 * i + 1]) + hi;
                        S.coef[2 * i] = -hr * sg;
                        S.coef[2 * i + 1] = -hi * sg;
                    }
                }
                __syncthreads();
                const double nn2 = cta_axpy(S.u, S.coef, j + 1, w, n, S.red, true);
                old = norm;
                norm = sqrt(nn2);
            }
            beta = norm;
            if (threadIdx.x == 0) {
                for (int i = 0; i <= j; i++) H[i + j * m] = cd{S.hacc[2 * i], S.hacc[2 * i + 1]};
            }
            const bool ok = norm != 0.0 && norm >= eta * old;
            if (!ok) {
                m_eff = j + 1;
                brokedown = true;
                __syncthreads();
                break;
            }
            if (threadIdx.x == 0) {
                if (j != m - 1) H[(j + 1) + j * m] = cd{norm, 0.0};
                S.sigma[j + 1] = 1.0 / norm;
            }
            __syncthreads();
        }
        // Hfull = [OldHfull 0; 0..0 oldbeta H] (inc/algo.h:303-328)
        const int nn = base + m_eff;
        for (int e = threadIdx.x; e < nn * nn; e += BT) {
            const int i = e % nn, j = e / nn;
            if (i >= base || j >= base) hfull[i + (size_t)j * a.hcap] = cd{0.0, 0.0};
        }
        __syncthreads();
        if (threadIdx.x == 0 && cycle > 1) hfull[base + (size_t)(base - 1) * a.hcap] = cd{oldbeta, 0.0};
        for (int e = threadIdx.x; e < m_eff * m_eff; e += BT) {
            const int i = e % m_eff, j = e / m_eff;
            hfull[(base + i) + (size_t)(base + j) * a.hcap] = H[i + j * m];
        }
        __syncthreads();
        cd *A = escr, *E = escr + (size_t)nn * nn, *ws = E + (size_t)nn * nn;
        const cd f{0.0, -t_real};
        for (int e = threadIdx.x; e < nn * nn; e += BT) {
            const int i = e % nn, j = e / nn;
            A[e] = cmul(f, hfull[i + (size_t)j * a.hcap]);
        }
        __syncthreads();
        expm_block(nn, A, E, ws, esmem);
        if (threadIdx.x == 0) {
            double sq = 0.0;
            for (int i = 0; i < m_eff; i++) {
                const cd e = E[base + i];
                sq += e.x * e.x + e.y * e.y;
                const double c = beta0 * S.sigma[i];
                S.coef[2 * i] = c * e.x;
                S.coef[2 * i + 1] = c * e.y;
            }
            S.nrm = sqrt(sq);
        }
        __syncthreads();
        cta_axpy(S.u, S.coef, m_eff, y, n, S.red, false);
        const double nrm = S.nrm;
        if ((a.max_restarts && cycle >= a.max_restarts) || brokedown || nrm < a.tol) break;
        // restart from v_m (swap_bufs(0, krydim), inc/algo.h:362)
        if (threadIdx.x == 0) {
            Cplx<float> *tmp = S.u[0];
            S.u[0] = S.u[m];
            S.u[m] = tmp;
            S.sigma[0] = S.sigma[m];
        }
        oldbeta = beta;
        __syncthreads();
    }
    cta_copy(psi, y, n);
    return true;
}

template <int B>
__device__ __noinline__ bool cta_otoc(const BatchProblem &P, const BatchArgs &a, char *slot, BatchShared &S,
                         unsigned char *stages, uint64_t *full, double *esmem, long &git,
                         int &applies, double &fr, double &fi) {
    const uint32_t n = 1u << P.len;
    Cplx<float> *psi = reinterpret_cast<Cplx<float> *>(slot + (size_t)(a.krydim + 2) * a.vec_stride);
    Cplx<float> *tmp = reinterpret_cast<Cplx<float> *>(slot + (size_t)(a.krydim + 3) * a.vec_stride);
    const double t = a.t;
    if (a.probe > 0) {   // tuning: H.psi products only
        cta_copy(psi, P.psi0, n);
        for (int r = 0; r < a.probe; r++) {
            if (!cta_apply<B>(P, (r & 1) ? tmp : psi, (r & 1) ? psi : tmp, 1.0, stages, full, git, a.err))
                return false;
            applies++;
        }
        return true;
    }
    cta_string(P.vx, P.vz, P.vcr, P.vci, P.psi0, psi, n);
    if (!cta_evolve<B>(P, psi, t, a, slot, S, stages, full, esmem, git, applies)) return false;
    cta_string(P.wx, P.wz, P.wcr, P.wci, psi, tmp, n);
    if (!cta_evolve<B>(P, tmp, -t, a, slot, S, stages, full, esmem, git, applies)) return false;
    cta_string(P.vx, P.vz, P.vcr, P.vci, tmp, psi, n);
    if (!cta_evolve<B>(P, psi, t, a, slot, S, stages, full, esmem, git, applies)) return false;
    cta_string(P.wx, P.wz, P.wcr, P.wci, psi, tmp, n);
    if (!cta_evolve<B>(P, tmp, -t, a, slot, S, stages, full, esmem, git, applies)) return false;
    cta_dot(P.psi0, tmp, n, S.red, fr, fi);
    return true;
}

__global__ void __launch_bounds__(BT, 1) k_batch_otoc(const BatchArgs a) {
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ BatchShared S;
    __shared__ __align__(8) uint64_t full[BST];
    unsigned char *stages = dsm;
    double *esmem = nullptr;
    if (threadIdx.x == 0) {
        for (int s = 0; s < BST; s++) mbar_init(&full[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    long git = 0;
    char *slot = a.ws + (size_t)blockIdx.x * a.ws_stride;
    while (true) {
        if (threadIdx.x == 0) S.item = atomicAdd(&a.counter[a.ti], 1);
        __syncthreads();
        const int item = S.item;
        __syncthreads();
        if (item >= a.nprob) break;
        const BatchProblem P = a.probs[item];
        // the expm's factor buffer sits after the largest ring in use
        esmem = reinterpret_cast<double *>(dsm + (size_t)BST * ((size_t)1 << P.B) * sizeof(Cplx<float>));
        int applies = 0;
        double fr = 0.0, fi = 0.0;
        bool ok = false;
        switch (P.B) {
            case 8: ok = cta_otoc<8>(P, a, slot, S, stages, full, esmem, git, applies, fr, fi); break;
            case 9: ok = cta_otoc<9>(P, a, slot, S, stages, full, esmem, git, applies, fr, fi); break;
            case 10: ok = cta_otoc<10>(P, a, slot, S, stages, full, esmem, git, applies, fr, fi); break;
            default: ok = cta_otoc<11>(P, a, slot, S, stages, full, esmem, git, applies, fr, fi); break;
        }
        if (!ok) break;
        if (threadIdx.x == 0) {
            a.F[((size_t)item * a.ntimes + a.ti) * 2] = fr;
            a.F[((size_t)item * a.ntimes + a.ti) * 2 + 1] = fi;
            a.applies[(size_t)item * a.ntimes + a.ti] = applies;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Host
// ---------------------------------------------------------------------------
static void split_string(uint64_t bits, int len, uint32_t &x, uint32_t &z) {
    x = z = 0;
    for (int i = 0; i < len; i++) {
        x |= (uint32_t)((bits >> (2 * i)) & 1) << i;
        z |= (uint32_t)((bits >> (2 * i + 1)) & 1) << i;
    }
}

void batch_free(BatchPlan &bp) {
    for (auto &p : bp.plans) plan_free(p);
    bp.plans.clear();
    if (bp.d_probs) cudaFree(bp.d_probs);
    if (bp.ws) cudaFree(bp.ws);
    if (bp.counter) cudaFree(bp.counter);
    if (bp.F) cudaFree(bp.F);
    if (bp.applies) cudaFree(bp.applies);
    if (bp.err) cudaFree(bp.err);
    if (bp.graph) cudaGraphExecDestroy(bp.graph);
    bp = BatchPlan{};
}

static size_t dyn_smem(int maxB, int hcap) {
    return (size_t)BST * ((size_t)1 << maxB) * sizeof(Cplx<float>) + (size_t)(2 * hcap + 64) * sizeof(double);
}

void batch_build(BatchPlan &bp, int nprob, const int *len, const int64_t *nterms,
                 const uint64_t *const *bits, const double *const *coeff, const uint64_t *wbits,
                 const double *wcoeff, const uint64_t *vbits, const double *vcoeff,
                 const void *const *psi0, const int *tile, int krydim, double tol,
                 int max_restarts, cudaStream_t st) {
    RP_REQUIRE(nprob >= 1, -2, "no problems in the batch");
    RP_REQUIRE(krydim >= 2 && krydim <= BMAXK, -2, "batched krydim must be in [2, 32]");
    RP_REQUIRE(max_restarts >= 1 && max_restarts <= 64, -2, "max_restarts must be in [1, 64]");
    batch_free(bp);
    bp.nprob = nprob;
    bp.krydim = krydim;
    bp.tol = tol;
    bp.max_restarts = max_restarts;
    bp.hcap = max_restarts * krydim;
    bp.plans.resize(nprob);
    std::vector<BatchProblem> probs(nprob);
    for (int p = 0; p < nprob; p++) {
        RP_REQUIRE(len[p] >= 8 && len[p] <= 30, -2, "batched problems need 8..30 qubits");
        RP_REQUIRE(psi0[p] && ((uintptr_t)psi0[p] & 15) == 0, -2, "psi0 must be 16-byte aligned");
        ApplyConfig cfg;
        int B = tile && tile[p] ? tile[p] : std::max(8, std::min(11, len[p] - 4));
        RP_REQUIRE(B >= 8 && B <= 11 && B <= len[p], -2, "batched tile exponent must be in [8, 11]");
        cfg.B = B;
        cfg.P = BT;
        cfg.stages = BST;
        cfg.allow_rows = false;
        plan_build(bp.plans[p], len[p], 1, bits[p], coeff[p], nterms[p], cfg);
        RP_REQUIRE(bp.plans[p].ngroups > 0, -2, "empty Hamiltonian in the batch");
        plan_upload(bp.plans[p]);
        BatchProblem &P = probs[p];
        P.terms = static_cast<const TermDesc<float> *>(bp.plans[p].d_terms);
        P.groups = bp.plans[p].d_groups;
        P.psi0 = static_cast<const Cplx<float> *>(psi0[p]);
        P.len = len[p];
        P.B = B;
        P.ntiles = bp.plans[p].ntiles;
        P.ngroups = bp.plans[p].ngroups;
        split_string(wbits[p], len[p], P.wx, P.wz);
        split_string(vbits[p], len[p], P.vx, P.vz);
        P.wcr = (float)wcoeff[2 * p];
        P.wci = (float)wcoeff[2 * p + 1];
        P.vcr = (float)vcoeff[2 * p];
        P.vci = (float)vcoeff[2 * p + 1];
        bp.maxB = std::max(bp.maxB, B);
        bp.maxlen = std::max(bp.maxlen, len[p]);
    }
    // largest problems first (they take longest)
    bp.order.resize(nprob);
    for (int p = 0; p < nprob; p++) bp.order[p] = p;
    std::stable_sort(bp.order.begin(), bp.order.end(),
                     [&](int x, int y) { return probs[x].len > probs[y].len; });
    for (int i = 0; i < nprob; i++) bp.probs.push_back(probs[bp.order[i]]);
    RP_CUDA(cudaMalloc((void **)&bp.d_probs, nprob * sizeof(BatchProblem)));
    RP_CUDA(cudaMemcpy(bp.d_probs, bp.probs.data(), nprob * sizeof(BatchProblem),
                       cudaMemcpyHostToDevice));
    // one workspace slot per resident CTA
    const size_t smem = dyn_smem(bp.maxB, bp.hcap);
    RP_CUDA(cudaFuncSetAttribute(k_batch_otoc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    int per_sm = 0;
    RP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_otoc, BT, smem));
    RP_REQUIRE(per_sm >= 1, -2, "batched kernel does not fit on an SM");
    bp.nslots = std::min(nprob, per_sm * num_sms());
    bp.vec_stride = (((size_t)1 << bp.maxlen) * sizeof(Cplx<float>) + 255) & ~(size_t)255;
    const size_t small = ((size_t)krydim * krydim + (size_t)bp.hcap * bp.hcap +
                          10 * (size_t)bp.hcap * bp.hcap) * sizeof(cd);
    bp.ws_stride = (((size_t)(krydim + 4) * bp.vec_stride + small) + 255) & ~(size_t)255;
    cudaError_t e = cudaMalloc(&bp.ws, bp.ws_stride * bp.nslots);
    if (e != cudaSuccess) {
        cudaGetLastError();
        batch_free(bp);
        throw Error{-4, "device out of memory for the batched workspace"};
    }
    RP_CUDA(cudaMalloc((void **)&bp.err, sizeof(unsigned)));
    RP_CUDA(cudaMemset(bp.err, 0, sizeof(unsigned)));
    (void)st;
}

double batch_probe(BatchPlan &bp, int napplies, cudaStream_t st) {
    RP_REQUIRE(napplies >= 1 && napplies <= 64, -2, "napplies must be in [1, 64]");
    const double zero = 0.0;
    BatchArgs a{};
    if (bp.ntimes_cap < 1) {
        RP_CUDA(cudaMalloc((void **)&bp.counter, sizeof(int)));
        RP_CUDA(cudaMalloc((void **)&bp.F, (size_t)bp.nprob * 2 * sizeof(double)));
        RP_CUDA(cudaMalloc((void **)&bp.applies, (size_t)bp.nprob * sizeof(int)));
        bp.ntimes_cap = 1;
    }
    a.probs = bp.d_probs;
    a.nprob = bp.nprob;
    a.krydim = bp.krydim;
    a.max_restarts = bp.max_restarts;
    a.ntimes = 1;
    a.hcap = bp.hcap;
    a.tol = bp.tol;
    a.t = zero;
    a.probe = napplies;
    a.F = bp.F;
    a.applies = bp.applies;
    a.ws = static_cast<char *>(bp.ws);
    a.ws_stride = bp.ws_stride;
    a.vec_stride = bp.vec_stride;
    a.counter = bp.counter;
    a.err = bp.err;
    const size_t smem = dyn_smem(bp.maxB, bp.hcap);
    cudaEvent_t e0, e1;
    RP_CUDA(cudaEventCreate(&e0));
    RP_CUDA(cudaEventCreate(&e1));
    RP_CUDA(cudaMemsetAsync(bp.err, 0, sizeof(unsigned), st));
    RP_CUDA(cudaMemsetAsync(bp.counter, 0, sizeof(int), st));
    RP_CUDA(cudaEventRecord(e0, st));
    k_batch_otoc<<<bp.nslots, BT, smem, st>>>(a);
    RP_CUDA(cudaGetLastError());
    RP_CUDA(cudaEventRecord(e1, st));
    unsigned herr = 0;
    RP_CUDA(cudaMemcpyAsync(&herr, bp.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    RP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    RP_REQUIRE(herr == 0, -5, "a device-side wait or bound failed in the batched kernel");
    return ms;
}

void batch_otoc(BatchPlan &bp, int ntimes, const double *times, double *F_host,
                int *applies_host, int use_graph, cudaStream_t st) {
    RP_REQUIRE(ntimes >= 1, -2, "no time points");
    if (ntimes > bp.ntimes_cap) {
        if (bp.counter) cudaFree(bp.counter);
        if (bp.F) cudaFree(bp.F);
        if (bp.applies) cudaFree(bp.applies);
        RP_CUDA(cudaMalloc((void **)&bp.counter, ntimes * sizeof(int)));
        RP_CUDA(cudaMalloc((void **)&bp.F, (size_t)bp.nprob * ntimes * 2 * sizeof(double)));
        RP_CUDA(cudaMalloc((void **)&bp.applies, (size_t)bp.nprob * ntimes * sizeof(int)));
        bp.ntimes_cap = ntimes;
        if (bp.graph) cudaGraphExecDestroy(bp.graph);
        bp.graph = nullptr;
    }
    const size_t smem = dyn_smem(bp.maxB, bp.hcap);
    BatchArgs a{};
    a.probs = bp.d_probs;
    a.nprob = bp.nprob;
    a.krydim = bp.krydim;
    a.max_restarts = bp.max_restarts;
    a.ntimes = ntimes;
    a.hcap = bp.hcap;
    a.tol = bp.tol;
    a.F = bp.F;
    a.applies = bp.applies;
    a.ws = static_cast<char *>(bp.ws);
    a.ws_stride = bp.ws_stride;
    a.vec_stride = bp.vec_stride;
    a.counter = bp.counter;
    a.err = bp.err;
    auto enqueue = [&](cudaStream_t s) {
        RP_CUDA(cudaMemsetAsync(bp.counter, 0, ntimes * sizeof(int), s));
        for (int k = 0; k < ntimes; k++) {
            a.t = times[k];
            a.ti = k;
            k_batch_otoc<<<bp.nslots, BT, smem, s>>>(a);
            RP_CUDA(cudaGetLastError());
        }
    };
    RP_CUDA(cudaMemsetAsync(bp.err, 0, sizeof(unsigned), st));
    if (use_graph) {
        const bool same = bp.graph && bp.graph_times == std::vector<double>(times, times + ntimes);
        if (!same) {
            if (bp.graph) cudaGraphExecDestroy(bp.graph);
            bp.graph = nullptr;
            cudaStream_t cs;
            RP_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            cudaGraph_t g;
            RP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            enqueue(cs);
            RP_CUDA(cudaStreamEndCapture(cs, &g));
            RP_CUDA(cudaGraphInstantiate(&bp.graph, g, 0));
            cudaGraphDestroy(g);
            cudaStreamDestroy(cs);
            bp.graph_times.assign(times, times + ntimes);
        }
        RP_CUDA(cudaGraphLaunch(bp.graph, st));
    } else {
        enqueue(st);
    }
    std::vector<double> F((size_t)bp.nprob * ntimes * 2);
    std::vector<int> ap((size_t)bp.nprob * ntimes);
    unsigned herr = 0;
    RP_CUDA(cudaMemcpyAsync(F.data(), bp.F, F.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaMemcpyAsync(ap.data(), bp.applies, ap.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaMemcpyAsync(&herr, bp.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
    RP_REQUIRE(herr == 0, -5, "a device-side wait or bound failed in the batched kernel");
    for (int i = 0; i < bp.nprob; i++) {
        const int p = bp.order[i];
        for (int k = 0; k < ntimes; k++) {
            if (F_host) {
                F_host[((size_t)p * ntimes + k) * 2] = F[((size_t)i * ntimes + k) * 2];
                F_host[((size_t)p * ntimes + k) * 2 + 1] = F[((size_t)i * ntimes + k) * 2 + 1];
            }
            if (applies_host) applies_host[(size_t)p * ntimes + k] = ap[(size_t)i * ntimes + k];
        }
    }
}

}  // namespace rp
