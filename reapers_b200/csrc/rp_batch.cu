// Batched OTOC on one GPU: one persistent launch per time step and team size.
//
// Work item = one problem (a disorder realisation x random state, any qubit
// count).  A team -- a thread-block cluster of C CTAs (C = 1..16, chosen per
// problem size) -- takes items from an atomic queue and runs the whole OTOC
// point for its item, in the operator order of
// examples/simple-syk-krylov.cc:42-57 at beta = 0:
//     psi = V psi0; e^{-iHt}; W; e^{iHt}; V; e^{-iHt}; W; e^{iHt}; <psi0|psi>,
// each evolve being the reference's restarted Krylov (inc/algo.h:77-173,
// 267-365: same pass criterion, breakdown rule, Hfull growth and ||Hexp0||
// test).  The team splits every vector pass: CTA r owns elements
// [r n / C, (r + 1) n / C) of copies, Pauli strings, projections and
// updates, and output tiles r, r + C, ... of H.psi, so the team's tiles in
// flight form a window of C consecutive tiles whose shared source tiles
// come from L2.  H.psi streams 2^B-element source tiles through a 4-stage
// bulk-copy ring per CTA (B per problem, chosen by the autotuner), whose
// source reads carry an L2 evict-last hint.
// Reductions: every CTA publishes its partial sums (and an ok flag) in
// shared memory, the cluster barrier (release/acquire at cluster scope)
// separates phases, and every CTA adds the C partials in rank order through
// distributed shared memory -- so all CTAs hold bit-identical sums and take
// identical control decisions.  The small FP64 work (H, Hfull, Pade-13 exp)
// is done by CTA 0 and its coefficients read by the others the same way.
// Teams never wait on other teams.  Vectors are FP32 (the mixed-precision
// form); everything else FP64.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>

#include "rp_batch.cuh"
#include "rp_expm_impl.cuh"
#include "rp_rows_dev.cuh"

namespace cg = cooperative_groups;

namespace rp {

constexpr int BT = 256;          // threads per CTA
constexpr int BNW = BT / 32;
constexpr int BST = 4;           // shared-memory stages of the H.psi ring
constexpr int BMAXK = 32;        // largest krydim of the batched form
constexpr int RB = 12;           // row-tile exponent: 256 rows x 16 complex64
constexpr unsigned RTILE = 256u * 128u;   // bytes of a row tile
constexpr int RS = 2;            // stages of the row-tile ring
constexpr int RMAXT = 512;       // largest row-kernel term / group tables in shared memory

struct BatchArgs {
    const BatchProblem *probs;   // this launch's problems (one team size)
    int nprob, out_base, krydim, max_restarts, ti, ntimes, hcap;
    int probe;          // > 0: only `probe` H.psi products per item (tuning)
    double t, tol;
    double *F;
    int *applies;
    char *ws;
    size_t ws_stride, vec_stride;
    int *counter;
    unsigned *err;
    const CUtensorMap *maps;     // [team slot][vector] 2-D TMA maps (row-tile problems)
    int nvec;                    // vectors per slot
    size_t stage_bytes;          // ring stages (a multiple of 1024)
    size_t table_bytes;          // row-kernel tables (0 without row-tile problems)
    size_t rterm_bytes;          // the term table's share of table_bytes
};

struct BatchShared {
    double red[2 * BNW];
    double part[2][4];            // published partials: [buffer][re, im, ok, -]
    double gpart[2][16];          // published grouped projections: [buffer][re, im x 8]
    double gred[BNW][16];         // per-warp grouped sums
    double gres[16];              // team totals of the grouped projections
    double sigma[BMAXK + 1];
    double hacc[2 * (BMAXK + 1)];
    double coef[2 * (BMAXK + 1)];
    double nrm;
    Cplx<float> *u[BMAXK + 1];
    int ui[BMAXK + 1];            // slot vector index of u[i] (its TMA map)
    int item;
    int pbuf;                     // which part[] buffer the next reduction uses
    int abort;                    // the ring's producer gave up (bounded wait)
};

__device__ __forceinline__ void proxy_fence_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// The team of one problem: cluster rank and size, and this CTA's share of
// an n-element pass.
struct Team {
    unsigned rank, size;
    __device__ uint32_t lo(uint32_t n) const { return (uint32_t)(((uint64_t)n * rank) / size); }
    __device__ uint32_t hi(uint32_t n) const { return (uint32_t)(((uint64_t)n * (rank + 1)) / size); }
};

__device__ __forceinline__ void team_sync() { cg::this_cluster().sync(); }

// Fixed-order sums over the CTA, broadcast to every thread of the CTA.
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

// Team-wide fixed-order sums of (a, b) and AND of ok, identical in every
// CTA.  One cluster barrier; the two partial buffers alternate, so a buffer
// is rewritten only after every CTA has passed the barrier that follows its
// reads.
__device__ bool team_reduce(const Team &tm, double &a, double &b, bool ok, BatchShared &S) {
    cta_sum2(a, b, S.red);
    const int buf = S.pbuf;
    if (threadIdx.x == 0) {
        S.part[buf][0] = a;
        S.part[buf][1] = b;
        S.part[buf][2] = ok ? 1.0 : 0.0;
    }
    team_sync();
    cg::cluster_group cl = cg::this_cluster();
    CompSum ca, cb;
    bool all = true;
    for (unsigned r = 0; r < tm.size; r++) {
        const double *pr = cl.map_shared_rank(&S.part[buf][0], r);
        ca.add(pr[0]);
        cb.add(pr[1]);
        all = all && pr[2] != 0.0;
    }
    a = ca.value();
    b = cb.value();
    __syncthreads();
    if (threadIdx.x == 0) S.pbuf = buf ^ 1;
    __syncthreads();
    return all;
}

__device__ __forceinline__ bool team_and(const Team &tm, bool ok, BatchShared &S) {
    double a = 0.0, b = 0.0;
    return team_reduce(tm, a, b, ok, S);
}

// <a|b> over n elements.
__device__ __noinline__ void team_dot(const Team &tm, const Cplx<float> *a, const Cplx<float> *b, uint32_t n,
                         BatchShared &S, double &re, double &im) {
    double sr = 0.0, si = 0.0;
    for (uint32_t k = tm.lo(n) + threadIdx.x; k < tm.hi(n); k += BT) {
        const Cplx<float> x = a[k], y = b[k];
        sr = fma((double)x.x, (double)y.x, fma((double)x.y, (double)y.y, sr));
        si = fma((double)x.x, (double)y.y, fma(-(double)x.y, (double)y.x, si));
    }
    team_reduce(tm, sr, si, true, S);
    re = sr;
    im = si;
}

// Basis-vector reads of the projection and update passes.  From 2^17
// elements per state on they stream through L2 with evict-first priority
// (ld.global.cs), which keeps the H.psi source tiles resident: measured
// +7 % (18 qubits) and +5 % (20 qubits) batched OTOC throughput, while on
// 16-qubit states, whose basis is re-read from L2, plain loads are 4.5 %
// faster.  The choice is made once per pass (a template argument): a
// run-time test inside the unrolled loads cost 15 % at every size.
constexpr uint32_t STREAM_MIN = 1u << 17;
template <bool STREAM>
__device__ __forceinline__ float4 ld_basis(const Cplx<float> *p) {
    if constexpr (STREAM) {
        return __ldcs(reinterpret_cast<const float4 *>(p));
    } else {
        return *reinterpret_cast<const float4 *>(p);
    }
}

constexpr int TG = 8;   // basis vectors projected (or added) per pass over w

// The passes below move 16-byte packets (two complex64 elements) per load:
// a team's range of every vector starts at an even element (ranges are
// n / C elements, n >= 2^8, C <= 16) and the workspace vectors are 16-byte
// aligned.  Each thread keeps up to TG + 1 packet loads in flight per step.

// This thread's FP64 partial sums of <u_i|w>, i in [i0, i0 + ng).
template <bool STREAM>
__device__ __forceinline__ void dots_pass(const Team &tm, Cplx<float> *const *u, int i0, int ng,
                                          const Cplx<float> *w, uint32_t n, double (&sr)[TG],
                                          double (&si)[TG]) {
#pragma unroll
    for (int q = 0; q < TG; q++) sr[q] = si[q] = 0.0;
    const uint32_t lo = tm.lo(n) >> 1, hi = tm.hi(n) >> 1;
    const float4 *w4 = reinterpret_cast<const float4 *>(w);
    for (uint32_t k = lo + threadIdx.x; k < hi; k += BT) {
        const float4 y = w4[k];
#pragma unroll
        for (int q = 0; q < TG; q++) {
            if (q < ng) {
                const float4 x = ld_basis<STREAM>(&u[i0 + q][2 * k]);
                double a = sr[q], b = si[q];
                a = fma((double)x.x, (double)y.x, fma((double)x.y, (double)y.y, a));
                b = fma((double)x.x, (double)y.y, fma(-(double)x.y, (double)y.x, b));
                a = fma((double)x.z, (double)y.z, fma((double)x.w, (double)y.w, a));
                b = fma((double)x.z, (double)y.w, fma(-(double)x.w, (double)y.z, b));
                sr[q] = a;
                si[q] = b;
            }
        }
    }
}

// <u_i|w> for i in [i0, i0 + ng), ng <= TG, in one pass over w: per-thread
// FP64 sums, fixed-order combination over the CTA's warps and then over the
// team's CTAs (all CTAs hold the same bits).  One cluster barrier.
__device__ __noinline__ void team_dots(const Team &tm, Cplx<float> *const *u, int i0, int ng,
                                       const Cplx<float> *w, uint32_t n, BatchShared &S,
                                       double *re, double *im) {
    double sr[TG], si[TG];
    if (n >= STREAM_MIN)
        dots_pass<true>(tm, u, i0, ng, w, n, sr, si);
    else
        dots_pass<false>(tm, u, i0, ng, w, n, sr, si);
    // CTA: warp sums, then the warps in order
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < TG; q++) {
        if (q >= ng) break;
        const double a = warp_sum(sr[q]), b = warp_sum(si[q]);
        if (lane == 0) {
            S.gred[warp][2 * q] = a;
            S.gred[warp][2 * q + 1] = b;
        }
    }
    __syncthreads();
    const int buf = S.pbuf;
    if (threadIdx.x < 2 * ng) {
        CompSum c;
        for (int wi = 0; wi < BNW; wi++) c.add(S.gred[wi][threadIdx.x]);
        S.gpart[buf][threadIdx.x] = c.value();
    }
    team_sync();
    cg::cluster_group cl = cg::this_cluster();
    if (threadIdx.x < 2 * ng) {
        CompSum c;
        for (unsigned r = 0; r < tm.size; r++) c.add(cl.map_shared_rank(&S.gpart[buf][0], r)[threadIdx.x]);
        S.gres[threadIdx.x] = c.value();
    }
    __syncthreads();
    for (int q = 0; q < ng; q++) {
        re[q] = S.gres[2 * q];
        im[q] = S.gres[2 * q + 1];
    }
    __syncthreads();
    if (threadIdx.x == 0) S.pbuf = buf ^ 1;
    __syncthreads();
}

// Element passes end with the generic-proxy writes fenced for the bulk
// copies of later H.psi products, and a team barrier.
__device__ void team_copy(const Team &tm, Cplx<float> *dst, const Cplx<float> *src, uint32_t n) {
    for (uint32_t k = tm.lo(n) + threadIdx.x; k < tm.hi(n); k += BT) dst[k] = src[k];
    proxy_fence_global();
    team_sync();
}

__device__ void team_zero(const Team &tm, Cplx<float> *dst, uint32_t n) {
    for (uint32_t k = tm.lo(n) + threadIdx.x; k < tm.hi(n); k += BT) dst[k] = Cplx<float>{0.f, 0.f};
    proxy_fence_global();
    team_sync();
}

// out[k] = c (-1)^popc(z & (k ^ x)) in[k ^ x]  (SpinOp::apply, inc/ops.h:421-440)
__device__ void team_string(const Team &tm, uint32_t x, uint32_t z, float cr, float ci,
                            const Cplx<float> *in, Cplx<float> *out, uint32_t n) {
    for (uint32_t k = tm.lo(n) + threadIdx.x; k < tm.hi(n); k += BT) {
        const uint32_t m = k ^ x;
        const float s = (__popc(z & m) & 1) ? -1.f : 1.f;
        const Cplx<float> v = in[m];
        out[k] = Cplx<float>{s * (cr * v.x - ci * v.y), s * (cr * v.y + ci * v.x)};
    }
    proxy_fence_global();
    team_sync();
}

// This thread's share of w += sum_{i < nv} coef_i u_i; returns its part of
// ||w||^2.  The basis vectors are read in groups of TG independent packet
// loads (a run-time loop over single vectors left one load in flight).
template <bool STREAM>
__device__ __forceinline__ double axpy_pass(const Team &tm, Cplx<float> *const *u, const double *coef,
                                            int nv, Cplx<float> *w, uint32_t n) {
    double nrm = 0.0;
    const uint32_t lo = tm.lo(n) >> 1, hi = tm.hi(n) >> 1;
    float4 *w4 = reinterpret_cast<float4 *>(w);
    for (uint32_t k = lo + threadIdx.x; k < hi; k += BT) {
        const float4 w0 = w4[k];
        double ar = w0.x, ai = w0.y, br = w0.z, bi = w0.w;
        for (int i0 = 0; i0 < nv; i0 += TG) {
#pragma unroll
            for (int q = 0; q < TG; q++) {
                if (i0 + q < nv) {
                    const float4 v = ld_basis<STREAM>(&u[i0 + q][2 * k]);
                    const double cr = coef[2 * (i0 + q)], ci = coef[2 * (i0 + q) + 1];
                    ar = fma(cr, (double)v.x, fma(-ci, (double)v.y, ar));
                    ai = fma(cr, (double)v.y, fma(ci, (double)v.x, ai));
                    br = fma(cr, (double)v.z, fma(-ci, (double)v.w, br));
                    bi = fma(cr, (double)v.w, fma(ci, (double)v.z, bi));
                }
            }
        }
        const float4 r = make_float4((float)ar, (float)ai, (float)br, (float)bi);
        w4[k] = r;
        nrm = fma((double)r.x, (double)r.x, fma((double)r.y, (double)r.y, nrm));
        nrm = fma((double)r.z, (double)r.z, fma((double)r.w, (double)r.w, nrm));
    }
    return nrm;
}

// w += sum_{i < nv} coef_i u_i over the team; returns ||w||^2 (team-wide).
__device__ __noinline__ double team_axpy(const Team &tm, Cplx<float> *const *u, const double *coef, int nv,
                            Cplx<float> *w, uint32_t n, BatchShared &S) {
    double nrm = n >= STREAM_MIN ? axpy_pass<true>(tm, u, coef, nv, w, n)
                                 : axpy_pass<false>(tm, u, coef, nv, w, n);
    proxy_fence_global();
    double dummy = 0.0;
    team_reduce(tm, nrm, dummy, true, S);
    return nrm;
}

// out = scale * H in over the team's output tiles (rank, rank + C, ...),
// source tiles streamed through this CTA's shared-memory ring: full[s]
// completes when the bulk copy into stage s lands, empty[s] when every warp
// is done with it.  Thread 0 issues item i + BST - 1 after the warps released
// item i - 1, so warps run up to BST - 1 items apart without CTA barriers.
// git counts ring items across calls (stage = git % BST, parity (git/BST)&1).
// Returns false in every CTA of the team if a bounded wait gave up in any.
template <int B>
__device__ __noinline__ bool team_apply(const Team &tm, const BatchProblem &P, const Cplx<float> *in,
                                        Cplx<float> *out, double scale, unsigned char *stages,
                                        uint64_t *full, uint64_t *empty, long &git, BatchShared &S,
                                        unsigned *err) {
    constexpr int TILE = 1 << B, E = TILE / BT;
    constexpr unsigned TB = TILE * sizeof(Cplx<float>);
    const int my_tiles = P.ntiles > (int)tm.rank ? (P.ntiles - 1 - (int)tm.rank) / (int)tm.size + 1 : 0;
    const long total = (long)my_tiles * P.ngroups;
    const uint32_t t = threadIdx.x, lane = t & 31;
    const uint64_t keep = l2_policy_evict_last();   // the input is re-read once per group
    long issued = 0;                                // thread 0 only
    // item i into its stage, once the warps have released the stage's previous item
    auto issue = [&](long i) -> bool {
        const long gi = git + i;
        const int s = (int)(gi % BST);
        if (gi >= BST && !mbar_wait_bounded(&empty[s], (unsigned)(((gi / BST) - 1) & 1), err))
            return false;
        const int o = (int)tm.rank + (int)(i / P.ngroups) * (int)tm.size, g = (int)(i % P.ngroups);
        const uint32_t src = (uint32_t)o ^ P.groups[g].xh;
        mbar_arrive_expect_tx(&full[s], TB);
        bulk_g2s_hint(stages + (size_t)s * TB, in + ((size_t)src << B), TB, &full[s], keep);
        issued = i + 1;
        return true;
    };
    if (t == 0) {
        S.abort = 0;
        proxy_fence_global();
        for (long i = 0; i < BST - 1 && i < total; i++)
            if (!issue(i)) {
                S.abort = 1;
                break;
            }
    }
    __syncthreads();
    bool ok = true;
    float ar[E], ai[E];
    long it = 0;
    for (; it < total; ++it) {
        const long gi = git + it;
        const int s = (int)(gi % BST);
        const unsigned par = (unsigned)((gi / BST) & 1);
        if (t == 0 && it + BST - 1 < total && !S.abort)
            if (!issue(it + BST - 1)) S.abort = 1;
        const bool okw = mbar_wait_bounded(&full[s], par, err);
        if (!__all_sync(0xffffffffu, okw && *(volatile int *)&S.abort == 0)) {
            ok = false;
            break;
        }
        const int o = (int)tm.rank + (int)(it / P.ngroups) * (int)tm.size;
        const int g = (int)(it % P.ngroups);
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
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (g == P.ngroups - 1) {
            Cplx<float> *op = out + ((size_t)o << B) + t;
#pragma unroll
            for (int j = 0; j < E; j++)
                op[(size_t)j * BT] = Cplx<float>{(float)(scale * ar[j]), (float)(scale * ai[j])};
        }
    }
    if (!ok && t == 0) {
        // let every copy already issued land before the stages are reused
        for (long i = it; i < issued; i++)
            mbar_wait_bounded(&full[(git + i) % BST], (unsigned)(((git + i) / BST) & 1), err);
    }
    __syncthreads();
    git += total;
    proxy_fence_global();
    return team_and(tm, ok, S);
}

// Ring state of one CTA: shared-memory stages, full / empty barriers of the
// bulk-copy ring (tile loop) and of the row-tile ring, item counters, the
// problem's row tables in shared memory.
struct Ring {
    unsigned char *stages;   // 1024-byte aligned
    uint64_t *full, *empty, *rfull, *rempty;
    long git, rgit;
    const RowTerm<float> *sterms;
    const RowGroup *sgroups;
    RowTerm<float> *sterms_w;
    RowGroup *sgroups_w;
};

// out = scale * H in over the team's output tiles with the row kernel's
// layout: 4096-element tiles brought in by 2-D TMA copies with the 128-byte
// swizzle, thread t owns row t of the output tile and applies each term to
// its whole 128-byte row (the permutation inside the row is folded into the
// swizzled shared-memory address; eight compile-time cases of element
// swap, element sign and coefficient kind).  Ring protocol as team_apply.
__device__ __noinline__ bool team_apply_rows(const Team &tm, const BatchProblem &P,
                                             const CUtensorMap *map, Cplx<float> *out,
                                             double scale, Ring &R, BatchShared &S,
                                             unsigned *err) {
    constexpr int C = 16, LOGC = 4;
    const int ntiles = 1 << (P.len - RB);
    const int ng = P.rngroups;
    const int my_tiles = ntiles > (int)tm.rank ? (ntiles - 1 - (int)tm.rank) / (int)tm.size + 1 : 0;
    const long total = (long)my_tiles * ng;
    const uint32_t t = threadIdx.x, lane = t & 31;
    long issued = 0;
    auto issue = [&](long i) -> bool {
        const long gi = R.rgit + i;
        const int s = (int)(gi % RS);
        if (gi >= RS && !mbar_wait_bounded(&R.rempty[s], (unsigned)(((gi / RS) - 1) & 1), err))
            return false;
        const int o = (int)tm.rank + (int)(i / ng) * (int)tm.size, g = (int)(i % ng);
        const uint32_t src = (uint32_t)o ^ R.sgroups[g].xh;
        mbar_arrive_expect_tx(&R.rfull[s], RTILE);
        tma_load_2d(R.stages + (size_t)s * RTILE, map, 0, (int)(src * 256u), &R.rfull[s]);
        issued = i + 1;
        return true;
    };
    if (t == 0) {
        S.abort = 0;
        proxy_fence_global();
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
        for (long i = 0; i < RS - 1 && i < total; i++)
            if (!issue(i)) {
                S.abort = 1;
                break;
            }
    }
    __syncthreads();
    bool ok = true;
    Cplx<float> acc[C];
    long it = 0;
    for (; it < total; ++it) {
        const long gi = R.rgit + it;
        const int s = (int)(gi % RS);
        const unsigned par = (unsigned)((gi / RS) & 1);
        if (t == 0 && it + RS - 1 < total && !S.abort)
            if (!issue(it + RS - 1)) S.abort = 1;
        const bool okw = mbar_wait_bounded(&R.rfull[s], par, err);
        if (!__all_sync(0xffffffffu, okw && *(volatile int *)&S.abort == 0)) {
            ok = false;
            break;
        }
        const int o = (int)tm.rank + (int)(it / ng) * (int)tm.size;
        const int g = (int)(it % ng);
        if (g == 0) {
#pragma unroll
            for (int u = 0; u < C; u++) acc[u].x = acc[u].y = 0.f;
        }
        const RowGroup gd = R.sgroups[g];
        const uint32_t src_hi = ((uint32_t)o ^ gd.xh) << RB;
        const uint32_t tile = smem_u32(R.stages + (size_t)s * RTILE);
        for (uint32_t k = gd.first; k < gd.first + gd.count; ++k) {
            const uint4 d0 = *reinterpret_cast<const uint4 *>(&R.sterms[k]);
            const uint32_t cs = d0.x, z = d0.y, jc = d0.z;
            const uint32_t sr = t ^ (cs & 0xFFu);
            const uint32_t xq = (cs >> 8) & 7u;
            const uint32_t s0 = (uint32_t)(__popc(z & (src_hi | (sr << LOGC))) & 1);
            float c0 = __uint_as_float(d0.w);
            if (s0) c0 = -c0;
            const uint32_t rq = (tile + sr * 128u) | ((xq ^ (sr & 7u)) << 4);
            switch ((cs >> 11) & 7u) {
                case 0: chunk_case<float, 0>(acc, rq, c0, jc); break;
                case 1: chunk_case<float, 1>(acc, rq, c0, jc); break;
                case 2: chunk_case<float, 2>(acc, rq, c0, jc); break;
                case 3: chunk_case<float, 3>(acc, rq, c0, jc); break;
                case 4: chunk_case<float, 4>(acc, rq, c0, jc); break;
                case 5: chunk_case<float, 5>(acc, rq, c0, jc); break;
                case 6: chunk_case<float, 6>(acc, rq, c0, jc); break;
                default: chunk_case<float, 7>(acc, rq, c0, jc); break;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&R.rempty[s]);
        if (g == ng - 1) {
            float4 *orow = reinterpret_cast<float4 *>(out + ((size_t)o << RB) + (size_t)t * C);
#pragma unroll
            for (int p = 0; p < 8; p++)
                orow[p] = make_float4((float)(scale * acc[2 * p].x), (float)(scale * acc[2 * p].y),
                                      (float)(scale * acc[2 * p + 1].x),
                                      (float)(scale * acc[2 * p + 1].y));
        }
    }
    if (!ok && t == 0) {
        for (long i = it; i < issued; i++)
            mbar_wait_bounded(&R.rfull[(R.rgit + i) % RS], (unsigned)(((R.rgit + i) / RS) & 1), err);
    }
    __syncthreads();
    R.rgit += total;
    proxy_fence_global();
    return team_and(tm, ok, S);
}

// H.psi of slot vector `in_idx` (pointer `in`) into out, by the problem's loop.
template <int B>
__device__ __forceinline__ bool team_H(const Team &tm, const BatchProblem &P, const BatchArgs &a,
                                       int in_idx, const Cplx<float> *in, Cplx<float> *out,
                                       double scale, Ring &R, BatchShared &S) {
    if (P.rows) {
        const unsigned team_id = blockIdx.x / tm.size;
        return team_apply_rows(tm, P, a.maps + (size_t)team_id * a.nvec + in_idx, out, scale, R,
                               S, a.err);
    }
    return team_apply<B>(tm, P, in, out, scale, R.stages, R.full, R.empty, R.git, S, a.err);
}

// psi <- exp(-i t H) psi by the reference's restarted Krylov, run by a team.
template <int B>
__device__ bool team_evolve(const Team &tm, const BatchProblem &P, Cplx<float> *psi,
                            double t_real, const BatchArgs &a, char *slot, BatchShared &S,
                            Ring &R, double *esmem, int &applies) {
    if (t_real == 0.0) return true;   // State::evolve returns at t = beta = 0
    const uint32_t n = 1u << P.len;
    const int m = a.krydim;
    const double eta = 1.0 / sqrt(2.0);
    const bool lead = tm.rank == 0;
    Cplx<float> *y = reinterpret_cast<Cplx<float> *>(slot + (size_t)(m + 1) * a.vec_stride);
    cd *H = reinterpret_cast<cd *>(slot + (size_t)(m + 4) * a.vec_stride);
    cd *hfull = H + m * m;
    cd *escr = hfull + (size_t)a.hcap * a.hcap;
    if (threadIdx.x == 0)
        for (int i = 0; i <= m; i++) {
            S.u[i] = reinterpret_cast<Cplx<float> *>(slot + (size_t)i * a.vec_stride);
            S.ui[i] = i;
        }
    __syncthreads();
    double b2, dummy;
    team_dot(tm, psi, psi, n, S, b2, dummy);
    const double beta0 = sqrt(b2);
    if (beta0 == 0.0) return true;
    for (uint32_t k = tm.lo(n) + threadIdx.x; k < tm.hi(n); k += BT) {
        S.u[0][k] = psi[k];
        y[k] = Cplx<float>{0.f, 0.f};
    }
    proxy_fence_global();
    if (threadIdx.x == 0) S.sigma[0] = 1.0 / beta0;
    team_sync();
    double oldbeta = 0.0, beta = 0.0;
    for (int cycle = 1;; cycle++) {
        const int base = (cycle - 1) * m;
        if (base + m > a.hcap) {   // bounded by max_restarts on the host; defensive
            if (lead && threadIdx.x == 0) atomicOr(a.err, DEV_ERR_BOUNDS);
            return false;          // every CTA of the team takes this branch
        }
        if (lead) {
            for (int e = threadIdx.x; e < 2 * m * m; e += BT) reinterpret_cast<double *>(H)[e] = 0.0;
        }
        __syncthreads();
        int m_eff = m;
        bool brokedown = false;
        for (int j = 0; j < m; j++) {
            Cplx<float> *w = S.u[j + 1];
            if (!team_H<B>(tm, P, a, S.ui[j], S.u[j], w, S.sigma[j], R, S)) return false;
            applies++;
            double old = 1.0, norm = eta / 2;
            int niter = 0;
            while (niter < 3 && norm != 0.0 && norm < eta * old) {
                niter++;
                for (int i0 = 0; i0 <= j; i0 += TG) {
                    const int ng = j + 1 - i0 < TG ? j + 1 - i0 : TG;
                    double hr[TG], hi[TG];
                    team_dots(tm, S.u, i0, ng, w, n, S, hr, hi);
                    if (threadIdx.x == 0) {
                        for (int q = 0; q < ng; q++) {
                            const int i = i0 + q;
                            const double sg = S.sigma[i];
                            const double r = hr[q] * sg, m_ = hi[q] * sg;
                            S.hacc[2 * i] = (niter == 1 ? 0.0 : S.hacc[2 * i]) + r;
                            S.hacc[2 * i + 1] = (niter == 1 ? 0.0 : S.hacc[2 * i + 1]) + m_;
                            S.coef[2 * i] = -r * sg;
                            S.coef[2 * i + 1] = -m_ * sg;
                        }
                    }
                }
                __syncthreads();
                const double nn2 = team_axpy(tm, S.u, S.coef, j + 1, w, n, S);
                old = norm;
                norm = sqrt(nn2);
            }
            beta = norm;
            if (lead && threadIdx.x == 0) {
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
                if (lead && j != m - 1) H[(j + 1) + j * m] = cd{norm, 0.0};
                S.sigma[j + 1] = 1.0 / norm;
            }
            __syncthreads();
        }
        const int nn = base + m_eff;
        if (lead) {
            // Hfull = [OldHfull 0; 0..0 oldbeta H] (inc/algo.h:303-328)
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
        }
        // the leader's coefficients and convergence norm to the whole team
        team_sync();
        if (!lead) {
            cg::cluster_group cl = cg::this_cluster();
            const double *lc = cl.map_shared_rank(&S.coef[0], 0);
            for (int i = threadIdx.x; i < 2 * m_eff; i += BT) S.coef[i] = lc[i];
            if (threadIdx.x == 0) S.nrm = *cl.map_shared_rank(&S.nrm, 0);
        }
        __syncthreads();
        team_axpy(tm, S.u, S.coef, m_eff, y, n, S);   // its barrier also ends the reads above
        const double nrm = S.nrm;
        if ((a.max_restarts && cycle >= a.max_restarts) || brokedown || nrm < a.tol) break;
        // restart from v_m (swap_bufs(0, krydim), inc/algo.h:362)
        if (threadIdx.x == 0) {
            Cplx<float> *tmp = S.u[0];
            S.u[0] = S.u[m];
            S.u[m] = tmp;
            const int ti = S.ui[0];
            S.ui[0] = S.ui[m];
            S.ui[m] = ti;
            S.sigma[0] = S.sigma[m];
        }
        oldbeta = beta;
        __syncthreads();
    }
    team_copy(tm, psi, y, n);
    return true;
}

template <int B>
__device__ __noinline__ bool team_otoc(const Team &tm, const BatchProblem &P, const BatchArgs &a,
                                       char *slot, BatchShared &S, Ring &R, double *esmem,
                                       int &applies, double &fr, double &fi) {
    const uint32_t n = 1u << P.len;
    Cplx<float> *psi = reinterpret_cast<Cplx<float> *>(slot + (size_t)(a.krydim + 2) * a.vec_stride);
    Cplx<float> *tmp = reinterpret_cast<Cplx<float> *>(slot + (size_t)(a.krydim + 3) * a.vec_stride);
    const double t = a.t;
    if (P.rows) {   // the problem's row tables into shared memory
        for (int i = threadIdx.x; i < P.rnterms; i += BT) R.sterms_w[i] = P.rterms[i];
        for (int i = threadIdx.x; i < P.rngroups; i += BT) R.sgroups_w[i] = P.rgroups[i];
        __syncthreads();
    }
    if (a.probe > 0) {   // tuning: H.psi products only
        team_copy(tm, psi, P.psi0, n);
        for (int r = 0; r < a.probe; r++) {
            const bool odd = r & 1;
            if (!team_H<B>(tm, P, a, odd ? a.krydim + 3 : a.krydim + 2, odd ? tmp : psi,
                           odd ? psi : tmp, 1.0, R, S))
                return false;
            applies++;
        }
        return true;
    }
    team_string(tm, P.vx, P.vz, P.vcr, P.vci, P.psi0, psi, n);
    if (!team_evolve<B>(tm, P, psi, t, a, slot, S, R, esmem, applies)) return false;
    team_string(tm, P.wx, P.wz, P.wcr, P.wci, psi, tmp, n);
    if (!team_evolve<B>(tm, P, tmp, -t, a, slot, S, R, esmem, applies)) return false;
    team_string(tm, P.vx, P.vz, P.vcr, P.vci, tmp, psi, n);
    if (!team_evolve<B>(tm, P, psi, t, a, slot, S, R, esmem, applies)) return false;
    team_string(tm, P.wx, P.wz, P.wcr, P.wci, psi, tmp, n);
    if (!team_evolve<B>(tm, P, tmp, -t, a, slot, S, R, esmem, applies)) return false;
    team_dot(tm, P.psi0, tmp, n, S, fr, fi);
    return true;
}

__global__ void __launch_bounds__(BT, 2) k_batch_otoc(const BatchArgs a) {
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ BatchShared S;
    __shared__ __align__(8) uint64_t full[BST];
    __shared__ __align__(8) uint64_t empty[BST];
    __shared__ __align__(8) uint64_t rfull[RS];
    __shared__ __align__(8) uint64_t rempty[RS];
    // dynamic shared memory: [ring stages, 1024-byte aligned for the 128-byte
    // swizzle][row-kernel term and group tables][the expm's factor buffer]
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(dsm) + 1023) & ~uintptr_t(1023));
    Ring R;
    R.stages = base;
    R.full = full;
    R.empty = empty;
    R.rfull = rfull;
    R.rempty = rempty;
    R.git = 0;
    R.rgit = 0;
    R.sterms_w = reinterpret_cast<RowTerm<float> *>(base + a.stage_bytes);
    R.sgroups_w = reinterpret_cast<RowGroup *>(base + a.stage_bytes + a.rterm_bytes);
    R.sterms = R.sterms_w;
    R.sgroups = R.sgroups_w;
    double *esmem = reinterpret_cast<double *>(base + a.stage_bytes + a.table_bytes);
    cg::cluster_group cl = cg::this_cluster();
    const Team tm{cl.block_rank(), cl.num_blocks()};
    if (threadIdx.x == 0) {
        for (int s = 0; s < BST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], BNW);
        }
        for (int s = 0; s < RS; s++) {
            mbar_init(&rfull[s], 1);
            mbar_init(&rempty[s], BNW);
        }
        fence_barrier_init();
        S.pbuf = 0;
        S.abort = 0;
    }
    __syncthreads();
    const unsigned team_id = blockIdx.x / tm.size;
    char *slot = a.ws + (size_t)team_id * a.ws_stride;
    while (true) {
        if (tm.rank == 0 && threadIdx.x == 0) S.item = atomicAdd(&a.counter[a.ti], 1);
        team_sync();
        const int item = *cl.map_shared_rank(&S.item, 0);
        team_sync();   // the leader rewrites S.item only after everyone read it
        if (item >= a.nprob) break;
        const BatchProblem P = a.probs[item];
        int applies = 0;
        double fr = 0.0, fi = 0.0;
        bool ok = false;
        switch (P.rows ? 11 : P.B) {
            case 8: ok = team_otoc<8>(tm, P, a, slot, S, R, esmem, applies, fr, fi); break;
            case 9: ok = team_otoc<9>(tm, P, a, slot, S, R, esmem, applies, fr, fi); break;
            case 10: ok = team_otoc<10>(tm, P, a, slot, S, R, esmem, applies, fr, fi); break;
            default: ok = team_otoc<11>(tm, P, a, slot, S, R, esmem, applies, fr, fi); break;
        }
        if (!ok) break;   // identical in every CTA of the team
        if (tm.rank == 0 && threadIdx.x == 0) {
            const size_t o = (size_t)(a.out_base + item) * a.ntimes + a.ti;
            a.F[o * 2] = fr;
            a.F[o * 2 + 1] = fi;
            a.applies[o] = applies;
        }
        __syncthreads();
    }
    // no CTA leaves while another may still read its shared memory
    team_sync();
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
    for (auto &r : bp.rplans) rowplan_free(r);
    bp.rplans.clear();
    if (bp.maps) cudaFree(bp.maps);
    if (bp.d_probs) cudaFree(bp.d_probs);
    if (bp.ws) cudaFree(bp.ws);
    if (bp.counter) cudaFree(bp.counter);
    if (bp.F) cudaFree(bp.F);
    if (bp.applies) cudaFree(bp.applies);
    if (bp.err) cudaFree(bp.err);
    if (bp.graph) cudaGraphExecDestroy(bp.graph);
    bp = BatchPlan{};
}

// Dynamic shared memory of a class: the ring stages (the larger of the two
// loops' rings in use), the row tables when a problem uses row tiles, the
// expm's factor buffer, and slack for the 1024-byte alignment.
static size_t stage_bytes(const BatchClass &c) {
    size_t b = 0;
    if (c.any_tiled) b = (size_t)BST * ((size_t)1 << c.maxB) * sizeof(Cplx<float>);
    if (c.any_rows) b = std::max(b, (size_t)RS * RTILE);
    return (b + 1023) & ~(size_t)1023;
}
// Row tables sized for the class's largest term and group lists, not for
// RMAXT: two CTAs per SM must leave room for the L1 share of the SM's
// unified L1 / shared memory.  A 1.4 KB larger footprint that pushed two
// CTAs from 194 to 197 KB (past the 196 KB carveout step) cost the row-tile
// H.psi loop 12-19 %.
static size_t rterm_bytes(const BatchClass &c) {
    return c.any_rows ? (size_t)c.maxrt * sizeof(RowTerm<float>) : 0;
}
static size_t table_bytes(const BatchClass &c) {
    return c.any_rows ? rterm_bytes(c) + (((size_t)c.maxrg * sizeof(RowGroup) + 15) & ~(size_t)15) : 0;
}
static size_t dyn_smem(const BatchClass &c, int hcap) {
    return 1024 + stage_bytes(c) + table_bytes(c) + (size_t)(2 * hcap + 64) * sizeof(double);
}

// Default team size: one CTA up to 2^16 elements, doubling per qubit above,
// at most 16 (the largest thread-block cluster).
static int default_team(int len) { return std::min(16, 1 << std::max(0, len - 16)); }

static cudaLaunchConfig_t class_config(const BatchClass &c, size_t smem, cudaStream_t st,
                                       cudaLaunchAttribute *attr) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(c.nslots * c.team), 1, 1);
    cfg.blockDim = dim3(BT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)c.team;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

void batch_build(BatchPlan &bp, int nprob, const int *len, const int64_t *nterms,
                 const uint64_t *const *bits, const double *const *coeff, const uint64_t *wbits,
                 const double *wcoeff, const uint64_t *vbits, const double *vcoeff,
                 const void *const *psi0, const int *tile, const int *team, int krydim, double tol,
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
    bp.rplans.resize(nprob);
    std::vector<BatchProblem> probs(nprob);
    std::vector<int> teams(nprob);
    for (int p = 0; p < nprob; p++) {
        RP_REQUIRE(len[p] >= 8 && len[p] <= 30, -2, "batched problems need 8..30 qubits");
        RP_REQUIRE(psi0[p] && ((uintptr_t)psi0[p] & 15) == 0, -2, "psi0 must be 16-byte aligned");
        RP_REQUIRE(nterms[p] >= 1, -2, "empty Hamiltonian in the batch");
        const int C = team && team[p] ? team[p] : default_team(len[p]);
        RP_REQUIRE(C == 1 || C == 2 || C == 4 || C == 8 || C == 16, -2,
                   "batched team size must be 1, 2, 4, 8 or 16");
        teams[p] = C;
        BatchProblem &P = probs[p];
        P = BatchProblem{};
        P.psi0 = static_cast<const Cplx<float> *>(psi0[p]);
        P.len = len[p];
        // row tiles (exponent 12) when asked for, or by default when the
        // state has a full tile and the tables fit in shared memory
        const int want = tile ? tile[p] : 0;
        RP_REQUIRE(want == 0 || (want >= 8 && want <= RB), -2,
                   "batched tile exponent must be in [8, 12]");
        bool rows = false;
        if ((want == RB || want == 0) && len[p] >= RB) {
            RowPlan &rp = bp.rplans[p];
            rowplan_build(rp, len[p], 1, bits[p], coeff[p], nterms[p], true);
            rows = rp.ok && rp.nterms <= RMAXT && (int)rp.groups.size() <= RMAXT;
            if (!rows) rowplan_free(rp), rp = RowPlan{};
        }
        RP_REQUIRE(want != RB || rows, -2,
                   "row tiles need >= 2^12 elements and at most 512 terms and groups");
        if (rows) {
            RowPlan &rp = bp.rplans[p];
            rowplan_upload(rp);
            P.rows = 1;
            P.rterms = static_cast<const RowTerm<float> *>(rp.d_terms);
            P.rgroups = rp.d_groups;
            P.rnterms = rp.nterms;
            P.rngroups = (int)rp.groups.size();
            P.B = RB;
            P.ntiles = rp.ntiles;
        } else {
            const int B = want ? want : std::max(8, std::min(11, len[p] - 4));
            RP_REQUIRE(B >= 8 && B <= 11 && B <= len[p], -2,
                       "batched tile exponent must be in [8, 11] and at most the qubit count");
            ApplyConfig cfg;
            cfg.B = B;
            cfg.P = BT;
            cfg.stages = BST;
            cfg.allow_rows = false;
            plan_build(bp.plans[p], len[p], 1, bits[p], coeff[p], nterms[p], cfg);
            RP_REQUIRE(bp.plans[p].ngroups > 0, -2, "empty Hamiltonian in the batch");
            plan_upload(bp.plans[p]);
            P.terms = static_cast<const TermDesc<float> *>(bp.plans[p].d_terms);
            P.groups = bp.plans[p].d_groups;
            P.B = B;
            P.ntiles = bp.plans[p].ntiles;
            P.ngroups = bp.plans[p].ngroups;
        }
        split_string(wbits[p], len[p], P.wx, P.wz);
        split_string(vbits[p], len[p], P.vx, P.vz);
        P.wcr = (float)wcoeff[2 * p];
        P.wci = (float)wcoeff[2 * p + 1];
        P.vcr = (float)vcoeff[2 * p];
        P.vci = (float)vcoeff[2 * p + 1];
    }
    // classes by team size (one launch each per time step), largest problems
    // first inside a class (they take longest)
    bp.order.resize(nprob);
    for (int p = 0; p < nprob; p++) bp.order[p] = p;
    std::stable_sort(bp.order.begin(), bp.order.end(), [&](int x, int y) {
        if (teams[x] != teams[y]) return teams[x] > teams[y];
        return probs[x].len > probs[y].len;
    });
    for (int i = 0; i < nprob; i++) bp.probs.push_back(probs[bp.order[i]]);
    for (int i = 0; i < nprob; i++) {
        const int p = bp.order[i];
        if (bp.classes.empty() || bp.classes.back().team != teams[p]) {
            BatchClass c;
            c.team = teams[p];
            c.first = i;
            bp.classes.push_back(c);
        }
        BatchClass &c = bp.classes.back();
        c.count++;
        if (probs[p].rows) {
            c.any_rows = true;
            c.maxrt = std::max(c.maxrt, probs[p].rnterms);
            c.maxrg = std::max(c.maxrg, probs[p].rngroups);
        } else {
            c.any_tiled = true;
            c.maxB = std::max(c.maxB, probs[p].B);
        }
        c.maxlen = std::max(c.maxlen, probs[p].len);
    }
    RP_CUDA(cudaMalloc((void **)&bp.d_probs, nprob * sizeof(BatchProblem)));
    RP_CUDA(cudaMemcpy(bp.d_probs, bp.probs.data(), nprob * sizeof(BatchProblem),
                       cudaMemcpyHostToDevice));
    // one workspace slot per resident team; the classes run one after the
    // other, so they share the allocation
    size_t smem_max = 0;
    for (auto &c : bp.classes) smem_max = std::max(smem_max, dyn_smem(c, bp.hcap));
    RP_REQUIRE(smem_max <= 227 * 1024, -2, "batched kernel shared memory above 227 KB");
    RP_CUDA(cudaFuncSetAttribute(k_batch_otoc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_max));
    RP_CUDA(cudaFuncSetAttribute(k_batch_otoc, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    size_t ws_bytes = 0;
    for (auto &c : bp.classes) {
        c.smem = dyn_smem(c, bp.hcap);
        cudaLaunchAttribute attr[1];
        BatchClass probe = c;
        probe.nslots = 1;
        cudaLaunchConfig_t cfg = class_config(probe, c.smem, st, attr);
        int nclusters = 0;
        RP_CUDA(cudaOccupancyMaxActiveClusters(&nclusters, k_batch_otoc, &cfg));
        RP_REQUIRE(nclusters >= 1, -2, "a batched team of this size does not fit on the GPU");
        c.nslots = std::min(nclusters, c.count);
        c.vec_stride = (((size_t)1 << c.maxlen) * sizeof(Cplx<float>) + 255) & ~(size_t)255;
        const size_t small = ((size_t)krydim * krydim + (size_t)bp.hcap * bp.hcap +
                              10 * (size_t)bp.hcap * bp.hcap) * sizeof(cd);
        c.ws_stride = (((size_t)(krydim + 4) * c.vec_stride + small) + 255) & ~(size_t)255;
        ws_bytes = std::max(ws_bytes, c.ws_stride * c.nslots);
    }
    cudaError_t e = cudaMalloc(&bp.ws, ws_bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        batch_free(bp);
        throw Error{-4, "device out of memory for the batched workspace"};
    }
    // 2-D TMA maps of every workspace vector of the classes with row-tile
    // problems (the map covers the slot's capacity, 2^maxlen elements)
    std::vector<CUtensorMap> maps;
    const int nvec = krydim + 4;
    for (auto &c : bp.classes) {
        c.map_base = (int)maps.size();
        if (!c.any_rows) continue;
        for (int sl = 0; sl < c.nslots; sl++)
            for (int v = 0; v < nvec; v++)
                maps.push_back(make_row_map(static_cast<char *>(bp.ws) + (size_t)sl * c.ws_stride +
                                                (size_t)v * c.vec_stride,
                                            c.maxlen, 1));
    }
    if (!maps.empty()) {
        RP_CUDA(cudaMalloc((void **)&bp.maps, maps.size() * sizeof(CUtensorMap)));
        RP_CUDA(cudaMemcpy(bp.maps, maps.data(), maps.size() * sizeof(CUtensorMap),
                           cudaMemcpyHostToDevice));
    }
    RP_CUDA(cudaMalloc((void **)&bp.err, sizeof(unsigned)));
    RP_CUDA(cudaMemset(bp.err, 0, sizeof(unsigned)));
}

static BatchArgs class_args(const BatchPlan &bp, const BatchClass &c, int ntimes) {
    BatchArgs a{};
    a.probs = bp.d_probs + c.first;
    a.nprob = c.count;
    a.out_base = c.first;
    a.krydim = bp.krydim;
    a.max_restarts = bp.max_restarts;
    a.ntimes = ntimes;
    a.hcap = bp.hcap;
    a.tol = bp.tol;
    a.F = bp.F;
    a.applies = bp.applies;
    a.ws = static_cast<char *>(bp.ws);
    a.ws_stride = c.ws_stride;
    a.vec_stride = c.vec_stride;
    a.err = bp.err;
    a.maps = c.any_rows ? bp.maps + c.map_base : nullptr;
    a.nvec = bp.krydim + 4;
    a.stage_bytes = stage_bytes(c);
    a.table_bytes = table_bytes(c);
    a.rterm_bytes = rterm_bytes(c);
    return a;
}

static void ensure_outputs(BatchPlan &bp, int ntimes) {
    if (ntimes <= bp.ntimes_cap) return;
    if (bp.counter) cudaFree(bp.counter);
    if (bp.F) cudaFree(bp.F);
    if (bp.applies) cudaFree(bp.applies);
    bp.counter = nullptr;
    bp.F = nullptr;
    bp.applies = nullptr;
    const size_t nc = bp.classes.size();
    RP_CUDA(cudaMalloc((void **)&bp.counter, nc * ntimes * sizeof(int)));
    RP_CUDA(cudaMalloc((void **)&bp.F, (size_t)bp.nprob * ntimes * 2 * sizeof(double)));
    RP_CUDA(cudaMalloc((void **)&bp.applies, (size_t)bp.nprob * ntimes * sizeof(int)));
    bp.ntimes_cap = ntimes;
    if (bp.graph) cudaGraphExecDestroy(bp.graph);
    bp.graph = nullptr;
}

double batch_probe(BatchPlan &bp, int napplies, cudaStream_t st) {
    RP_REQUIRE(napplies >= 1 && napplies <= 64, -2, "napplies must be in [1, 64]");
    ensure_outputs(bp, 1);
    cudaEvent_t e0, e1;
    RP_CUDA(cudaEventCreate(&e0));
    RP_CUDA(cudaEventCreate(&e1));
    RP_CUDA(cudaMemsetAsync(bp.err, 0, sizeof(unsigned), st));
    RP_CUDA(cudaMemsetAsync(bp.counter, 0, bp.classes.size() * sizeof(int), st));
    RP_CUDA(cudaEventRecord(e0, st));
    for (size_t ci = 0; ci < bp.classes.size(); ci++) {
        const BatchClass &c = bp.classes[ci];
        BatchArgs a = class_args(bp, c, 1);
        a.t = 0.0;
        a.ti = 0;
        a.probe = napplies;
        a.counter = bp.counter + ci;
        cudaLaunchAttribute attr[1];
        cudaLaunchConfig_t cfg = class_config(c, c.smem, st, attr);
        RP_CUDA(cudaLaunchKernelEx(&cfg, k_batch_otoc, a));
    }
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
    ensure_outputs(bp, ntimes);
    const size_t nc = bp.classes.size();
    auto enqueue = [&](cudaStream_t s) {
        RP_CUDA(cudaMemsetAsync(bp.counter, 0, nc * ntimes * sizeof(int), s));
        for (int k = 0; k < ntimes; k++) {
            for (size_t ci = 0; ci < nc; ci++) {
                const BatchClass &c = bp.classes[ci];
                BatchArgs a = class_args(bp, c, ntimes);
                a.t = times[k];
                a.ti = k;
                a.counter = bp.counter + ci * ntimes;
                cudaLaunchAttribute attr[1];
                cudaLaunchConfig_t cfg = class_config(c, c.smem, s, attr);
                RP_CUDA(cudaLaunchKernelEx(&cfg, k_batch_otoc, a));
            }
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
