// H.psi = sum_k c_k P_k psi for Pauli strings P_k = (x_k, z_k):
//   (H psi)[n] = sum_k c_k (-1)^popc(z_k & (n ^ x_k)) psi[n ^ x_k]
// (the per-element rule of SpinOp::apply, inc/ops.h:421-440, summed as in
// CPUImpl::apply_ops, inc/cpuimpl.h:739-754).
//
// Tiled design for sm_100a.  The output is cut into tiles of 2^B contiguous
// elements.  Terms are grouped by their high X-mask part xh = x >> B; every
// term of a group reads the same source tile (tile ^ xh), so one bulk copy
// of that tile into shared memory serves the whole group.  Per output tile a
// CTA streams the G distinct source tiles through a STAGES-deep pipeline
// (producer warp: cp.async.bulk + mbarrier transaction counts; P consumer
// threads: gather from shared memory, sign, FMA into registers) and writes
// the tile once.  HBM/L2 bytes per apply: (G + 1) * D * sizeof(element).
#include <algorithm>
#include <cstring>
#include <map>

#include "rp_apply.cuh"

namespace rp {

int num_sms() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        RP_CUDA(cudaGetDevice(&dev));
        RP_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    }
    return n;
}

template <typename Real>
static constexpr int stages_for(int B) {
    int bytes = (1 << B) * (int)sizeof(Cplx<Real>);
    int s = (3 * 65536) / bytes;
    return s < 2 ? 2 : (s > 8 ? 8 : s);
}

static size_t elem_size(int dtype) { return dtype == 2 ? 16 : 8; }

ApplyConfig default_config(int len, int dtype) {
    ApplyConfig c;
    if (len < 5) {
        c.direct = true;
        return c;
    }
    const int bmax = 12;
    // aim for at least ~256 output tiles so a single apply fills the GPU
    int B = len - 8;
    if (B > bmax) B = bmax;
    if (B < 5) B = 5;
    if (B > len) B = len;
    c.B = B;
    c.P = std::min(256, 1 << B);
    c.stages = dtype == 2 ? stages_for<double>(B) : stages_for<float>(B);
    return c;
}

template <typename Real>
static void build_terms(ApplyPlan &plan, const uint64_t *bits, const double *coeff,
                        int64_t nterms) {
    const ApplyConfig &cfg = plan.cfg;
    const int B = cfg.B, P = cfg.P;
    int logP = 0;
    while ((1 << logP) < P) logP++;
    const int E = (1 << B) / P;
    struct T {
        uint32_t x, z;
        double cr, ci;
        int64_t order;
    };
    std::vector<T> ts;
    ts.reserve(nterms);
    for (int64_t k = 0; k < nterms; k++) {
        uint32_t x = 0, z = 0;
        for (int i = 0; i < plan.len; i++) {
            x |= (uint32_t)((bits[k] >> (2 * i)) & 1) << i;
            z |= (uint32_t)((bits[k] >> (2 * i + 1)) & 1) << i;
        }
        ts.push_back({x, z, coeff[2 * k], coeff[2 * k + 1], k});
    }
    // group by the high X part; keep list order inside a group
    std::stable_sort(ts.begin(), ts.end(),
                     [B](const T &a, const T &b) { return (a.x >> B) < (b.x >> B); });
    plan.groups.clear();
    std::vector<TermDesc<Real>> out(ts.size());
    for (size_t k = 0; k < ts.size(); k++) {
        uint32_t xh = ts[k].x >> B;
        if (plan.groups.empty() || plan.groups.back().xh != xh)
            plan.groups.push_back({xh, (uint32_t)k, 0u, 0u});
        plan.groups.back().count++;
        TermDesc<Real> d;
        d.xl = ts[k].x & ((1u << B) - 1);
        d.z = ts[k].z;
        uint32_t zj = (ts[k].z >> logP) & (uint32_t)(E - 1);
        uint32_t xj = d.xl >> logP;
        uint32_t js = 0;
        for (int j = 0; j < E; j++) js |= (uint32_t)(__builtin_popcount(zj & (j ^ xj)) & 1) << j;
        d.jsign = js;
        d.cr = (Real)ts[k].cr;
        d.ci = (Real)ts[k].ci;
        d.kind = ts[k].ci == 0.0 ? COEFF_REAL : (ts[k].cr == 0.0 ? COEFF_IMAG : COEFF_COMPLEX);
        out[k] = d;
    }
    plan.term_bytes.resize(out.size() * sizeof(TermDesc<Real>));
    if (!out.empty()) memcpy(plan.term_bytes.data(), out.data(), plan.term_bytes.size());
}

template <typename Real>
struct DirectTerm {
    uint32_t x, z;
    Real cr, ci;
};

template <typename Real>
static void build_direct(ApplyPlan &plan, const uint64_t *bits, const double *coeff,
                         int64_t nterms) {
    std::vector<DirectTerm<Real>> out(nterms);
    for (int64_t k = 0; k < nterms; k++) {
        uint32_t x = 0, z = 0;
        for (int i = 0; i < plan.len; i++) {
            x |= (uint32_t)((bits[k] >> (2 * i)) & 1) << i;
            z |= (uint32_t)((bits[k] >> (2 * i + 1)) & 1) << i;
        }
        out[k] = {x, z, (Real)coeff[2 * k], (Real)coeff[2 * k + 1]};
    }
    plan.term_bytes.resize(out.size() * sizeof(DirectTerm<Real>));
    if (nterms) memcpy(plan.term_bytes.data(), out.data(), plan.term_bytes.size());
    plan.groups.clear();
}

void plan_build(ApplyPlan &plan, int len, int dtype, const uint64_t *bits,
                const double *coeff, int64_t nterms, const ApplyConfig &cfg) {
    RP_REQUIRE(len >= 1 && len <= 32, -2, "spin chain length must be in [1, 32]");
    RP_REQUIRE(dtype == 1 || dtype == 2, -2, "dtype must be RP_C64 (1) or RP_C128 (2)");
    RP_REQUIRE(nterms >= 0, -2, "number of terms must be non-negative");
    const uint64_t site_mask = len == 32 ? ~0ull : ((1ull << (2 * len)) - 1);
    for (int64_t k = 0; k < nterms; k++)
        RP_REQUIRE((bits[k] & ~site_mask) == 0, -2,
                   "a Pauli string acts on a site beyond the spin chain length");
    plan.len = len;
    plan.dtype = dtype;
    plan.cfg = cfg;
    plan.nterms = (int)nterms;
    const double D = std::ldexp(1.0, len);
    if (cfg.direct) {
        plan.ntiles = 0;
        if (dtype == 2) build_direct<double>(plan, bits, coeff, nterms);
        else build_direct<float>(plan, bits, coeff, nterms);
        plan.ngroups = 0;
        plan.alg_bytes = (double)(nterms + 1) * D * (double)elem_size(dtype);
        return;
    }
    RP_REQUIRE(cfg.B >= 5 && cfg.B <= 12 && cfg.B <= len, -2, "tile exponent out of range");
    plan.ntiles = 1 << (len - cfg.B);
    if (dtype == 2) build_terms<double>(plan, bits, coeff, nterms);
    else build_terms<float>(plan, bits, coeff, nterms);
    plan.ngroups = (int)plan.groups.size();
    plan.alg_bytes = (double)(plan.ngroups + 1) * D * (double)elem_size(dtype);
    plan.rows = RowPlan{};
    if (cfg.allow_rows) rowplan_build(plan.rows, len, dtype, bits, coeff, nterms, false, true);
    if (plan.rows.ok) plan.alg_bytes = plan.rows.alg_bytes_smem;
}

void plan_upload(ApplyPlan &plan) {
    plan_free(plan);
    size_t tb = plan.term_bytes.size();
    void *p = nullptr;
    RP_CUDA(cudaMalloc(&p, tb ? tb : 16));
    if (tb) RP_CUDA(cudaMemcpy(p, plan.term_bytes.data(), tb, cudaMemcpyHostToDevice));
    if (plan.cfg.direct) {
        plan.d_direct = p;
        return;
    }
    plan.d_terms = p;
    size_t gb = plan.groups.size() * sizeof(GroupDesc);
    RP_CUDA(cudaMalloc((void **)&plan.d_groups, gb ? gb : 16));
    if (gb) RP_CUDA(cudaMemcpy(plan.d_groups, plan.groups.data(), gb, cudaMemcpyHostToDevice));
    if (plan.rows.ok) rowplan_upload(plan.rows);
}

void plan_free(ApplyPlan &plan) {
    if (plan.d_terms) cudaFree(plan.d_terms);
    if (plan.d_groups) cudaFree(plan.d_groups);
    if (plan.d_direct) cudaFree(plan.d_direct);
    plan.d_terms = nullptr;
    plan.d_groups = nullptr;
    plan.d_direct = nullptr;
    rowplan_free(plan.rows);
}

int apply_grid(const ApplyPlan &plan) {
    if (plan.cfg.direct) return 1;
    if (plan.rows.ok) return plan.rows.window;
    return std::min(plan.ntiles, num_sms());
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
template <typename Real>
__device__ __forceinline__ Real flip_sign(Real c, uint32_t sb);
template <>
__device__ __forceinline__ float flip_sign<float>(float c, uint32_t sb) {
    return __uint_as_float(__float_as_uint(c) ^ sb);
}
template <>
__device__ __forceinline__ double flip_sign<double>(double c, uint32_t sb) {
    return __longlong_as_double(__double_as_longlong(c) ^ ((long long)sb << 32));
}

template <typename Real>
struct ApplyArgs {
    const Cplx<Real> *in;
    Cplx<Real> *out;
    const TermDesc<Real> *terms;
    const GroupDesc *groups;
    int ngroups;
    int ntiles;
    double alpha;
    const double *alpha_dev;
    int accumulate;
    const int *active;
    const Cplx<Real> *const *dot_vecs;
    int ndot;
    double *partials;
    unsigned *err;
};

constexpr int MAX_FUSED_DOTS = 64;

template <typename Real, int B, int P, int STAGES, bool DOTS>
__global__ void __launch_bounds__(P + 32, 1) k_apply_tiled(const ApplyArgs<Real> a) {
    constexpr int TILE = 1 << B;
    constexpr int E = TILE / P;
    constexpr int NW = P / 32;   // consumer warps
    constexpr unsigned TILE_BYTES = TILE * sizeof(Cplx<Real>);
    extern __shared__ __align__(1024) unsigned char smem[];
    Cplx<Real> *stage = reinterpret_cast<Cplx<Real> *>(smem);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * TILE_BYTES);
    uint64_t *empty = full + STAGES;
    // per-warp compensated partial projections: [NW][ndot] x {re.hi, re.lo, im.hi, im.lo}
    double *red = reinterpret_cast<double *>(empty + STAGES);
    __shared__ int s_abort;
    __shared__ long s_issued;

    if (a.active && *a.active == 0) return;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NW);
        }
        s_abort = 0;
        s_issued = 0;
        fence_barrier_init();
    }
    if (DOTS) {
        for (int i = tid; i < NW * a.ndot * 4; i += blockDim.x) red[i] = 0.0;
    }
    __syncthreads();

    const int ntile_iters =
        (int)blockIdx.x < a.ntiles ? (a.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const long total = (long)ntile_iters * a.ngroups;

    if (warp == NW) {
        // ---------------- producer ----------------
        if (lane == 0) {
            long it = 0;
            for (; it < total; ++it) {
                const int s = (int)(it % STAGES);
                const unsigned round = (unsigned)(it / STAGES);
                if (!mbar_wait_bounded(&empty[s], (round & 1u) ^ 1u, a.err)) {
                    atomicExch(&s_abort, 1);
                    break;
                }
                const long ti = it / a.ngroups;
                const int g = (int)(it - ti * a.ngroups);
                const uint32_t o = blockIdx.x + (uint32_t)ti * gridDim.x;
                const uint32_t src = o ^ __ldg(&a.groups[g].xh);
                mbar_arrive_expect_tx(&full[s], TILE_BYTES);
                bulk_g2s(stage + s * TILE, a.in + ((size_t)src << B), TILE_BYTES, &full[s]);
            }
            s_issued = it;
        }
    } else {
        // ---------------- consumers ----------------
        const uint32_t t = (uint32_t)tid;
        const double scale = a.alpha * (a.alpha_dev ? *a.alpha_dev : 1.0);
        long it = 0;
        bool ok = true;
        for (int ti = 0; ti < ntile_iters && ok; ++ti) {
            const uint32_t o = blockIdx.x + (uint32_t)ti * gridDim.x;
            Real ar[E], ai[E];
#pragma unroll
            for (int j = 0; j < E; j++) ar[j] = ai[j] = Real(0);
            for (int g = 0; g < a.ngroups; ++g, ++it) {
                const int s = (int)(it % STAGES);
                const unsigned round = (unsigned)(it / STAGES);
                if (!mbar_wait_bounded(&full[s], round & 1u, a.err)) {
                    ok = false;
                    break;
                }
                const Cplx<Real> *tile = stage + s * TILE;
                const GroupDesc gd = a.groups[g];
                const uint32_t src_hi = (o ^ gd.xh) << B;
                for (uint32_t k = gd.first; k < gd.first + gd.count; ++k) {
                    const uint4 td = __ldg(reinterpret_cast<const uint4 *>(&a.terms[k]));
                    const Real cr = __ldg(&a.terms[k].cr), ci = __ldg(&a.terms[k].ci);
                    const uint32_t xl = td.x, z = td.y, js = td.z, kind = td.w;
                    const uint32_t a0 = t ^ xl;
                    const uint32_t m0 = src_hi | (a0 & (uint32_t)(P - 1));
                    const uint32_t s0 = (uint32_t)(__popc(z & m0) & 1) << 31;
                    if (kind == COEFF_REAL) {
#pragma unroll
                        for (int j = 0; j < E; j++) {
                            const Cplx<Real> v = tile[a0 ^ (uint32_t)(j * P)];
                            const uint32_t sb = s0 ^ ((js << (31 - j)) & 0x80000000u);
                            const Real c = flip_sign(cr, sb);
                            ar[j] = fma(c, v.x, ar[j]);
                            ai[j] = fma(c, v.y, ai[j]);
                        }
                    } else if (kind == COEFF_IMAG) {
#pragma unroll
                        for (int j = 0; j < E; j++) {
                            const Cplx<Real> v = tile[a0 ^ (uint32_t)(j * P)];
                            const uint32_t sb = s0 ^ ((js << (31 - j)) & 0x80000000u);
                            const Real c = flip_sign(ci, sb);
                            ar[j] = fma(-c, v.y, ar[j]);
                            ai[j] = fma(c, v.x, ai[j]);
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < E; j++) {
                            const Cplx<Real> v = tile[a0 ^ (uint32_t)(j * P)];
                            const uint32_t sb = s0 ^ ((js << (31 - j)) & 0x80000000u);
                            const Real c1 = flip_sign(cr, sb), c2 = flip_sign(ci, sb);
                            ar[j] = fma(c1, v.x, fma(-c2, v.y, ar[j]));
                            ai[j] = fma(c1, v.y, fma(c2, v.x, ai[j]));
                        }
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[s]);
            }
            if (!ok) break;
            // write the tile (coalesced: each warp writes 32 consecutive elements per j)
            const size_t base = (size_t)o << B;
            Cplx<Real> w[E];
#pragma unroll
            for (int j = 0; j < E; j++) {
                Cplx<Real> *p = a.out + base + t + (size_t)j * P;
                Cplx<Real> r;
                r.x = (Real)(scale * (double)ar[j]);
                r.y = (Real)(scale * (double)ai[j]);
                if (a.accumulate) {
                    const Cplx<Real> old = *p;
                    r.x += old.x;
                    r.y += old.y;
                }
                *p = r;
                w[j] = r;
            }
            if (DOTS) {
                for (int i = 0; i < a.ndot; i++) {
                    const Cplx<Real> *u = a.dot_vecs[i] + base + t;
                    double sr = 0.0, si = 0.0;
#pragma unroll
                    for (int j = 0; j < E; j++) {
                        const Cplx<Real> uv = u[(size_t)j * P];
                        sr = fma((double)uv.x, (double)w[j].x, fma((double)uv.y, (double)w[j].y, sr));
                        si = fma((double)uv.x, (double)w[j].y, fma(-(double)uv.y, (double)w[j].x, si));
                    }
                    sr = warp_sum(sr);
                    si = warp_sum(si);
                    if (lane == 0) {
                        double *r = red + ((size_t)warp * a.ndot + i) * 4;
                        double s, e;
                        two_sum(r[0], sr, s, e);
                        r[0] = s;
                        r[1] += e;
                        two_sum(r[2], si, s, e);
                        r[2] = s;
                        r[3] += e;
                    }
                }
            }
        }
        if (!ok) atomicExch(&s_abort, 1);
    }
    __syncthreads();
    if (s_abort) {
        // wind down after a timed-out wait: at most STAGES copies can be in
        // flight (the producer reuses a stage only after it was released),
        // and they are the last STAGES issued.  Wait (bounded) for each so
        // none lands in shared memory after the CTA has exited.
        if (tid == 0) {
            const long issued = s_issued;
            for (long it = issued - STAGES; it < issued; ++it) {
                if (it < 0) continue;
                mbar_wait_bounded(&full[it % STAGES], (unsigned)((it / STAGES) & 1), a.err);
            }
        }
        return;
    }
    if (DOTS) {
        // fixed-order compensated sum over warps -> per-CTA partial
        for (int i = tid; i < a.ndot; i += blockDim.x) {
            CompSum re, im;
            for (int w = 0; w < NW; w++) {
                const double *r = red + ((size_t)w * a.ndot + i) * 4;
                re.add(r[0]);
                re.add(r[1]);
                im.add(r[2]);
                im.add(r[3]);
            }
            a.partials[((size_t)blockIdx.x * a.ndot + i) * 2 + 0] = re.value();
            a.partials[((size_t)blockIdx.x * a.ndot + i) * 2 + 1] = im.value();
        }
    }
}

// Tiny vectors (len < 5): one thread per element, terms in list order.
template <typename Real>
__global__ void k_apply_direct(const Cplx<Real> *in, Cplx<Real> *out,
                               const DirectTerm<Real> *terms, int nterms, uint32_t D,
                               double alpha, const double *alpha_dev, int accumulate,
                               const int *active) {
    if (active && *active == 0) return;
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= D) return;
    Real ar = 0, ai = 0;
    for (int k = 0; k < nterms; k++) {
        const DirectTerm<Real> tk = terms[k];
        const uint32_t m = n ^ tk.x;
        const Real sg = (__popc(tk.z & m) & 1) ? Real(-1) : Real(1);
        const Cplx<Real> v = in[m];
        const Real cr = sg * tk.cr, ci = sg * tk.ci;
        ar += cr * v.x - ci * v.y;
        ai += cr * v.y + ci * v.x;
    }
    const double scale = alpha * (alpha_dev ? *alpha_dev : 1.0);
    Cplx<Real> r;
    r.x = (Real)(scale * (double)ar);
    r.y = (Real)(scale * (double)ai);
    if (accumulate) {
        r.x += out[n].x;
        r.y += out[n].y;
    }
    out[n] = r;
}

// ---------------------------------------------------------------------------
// Launch dispatch
// ---------------------------------------------------------------------------
template <typename Real, int B, bool DOTS>
static void launch_tiled(const ApplyPlan &plan, const ApplyLaunch &l, cudaStream_t st) {
    constexpr int P = (1 << B) < 256 ? (1 << B) : 256;
    constexpr int STAGES = stages_for<Real>(B);
    constexpr size_t TILE_BYTES = (size_t)(1 << B) * sizeof(Cplx<Real>);
    const int NW = P / 32;
    size_t smem = STAGES * TILE_BYTES + 2 * STAGES * sizeof(uint64_t) +
                  (DOTS ? (size_t)NW * l.ndot * 4 * sizeof(double) : 0);
    auto kern = k_apply_tiled<Real, B, P, STAGES, DOTS>;
    static size_t attr_smem = 0;
    if (smem > attr_smem) {
        RP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        attr_smem = smem;
    }
    ApplyArgs<Real> a;
    a.in = static_cast<const Cplx<Real> *>(l.in);
    a.out = static_cast<Cplx<Real> *>(l.out);
    a.terms = static_cast<const TermDesc<Real> *>(plan.d_terms);
    a.groups = plan.d_groups;
    a.ngroups = plan.ngroups;
    a.ntiles = plan.ntiles;
    a.alpha = l.alpha;
    a.alpha_dev = l.alpha_dev;
    a.accumulate = l.accumulate;
    a.active = l.active;
    a.dot_vecs = reinterpret_cast<const Cplx<Real> *const *>(l.dot_vecs);
    a.ndot = l.ndot;
    a.partials = l.partials;
    a.err = l.err;
    const int grid = apply_grid(plan);
    kern<<<grid, P + 32, smem, st>>>(a);
    RP_CUDA(cudaGetLastError());
}

template <typename Real, bool DOTS>
static void dispatch_B(const ApplyPlan &plan, const ApplyLaunch &l, cudaStream_t st) {
    switch (plan.cfg.B) {
    case 5: launch_tiled<Real, 5, DOTS>(plan, l, st); break;
    case 6: launch_tiled<Real, 6, DOTS>(plan, l, st); break;
    case 7: launch_tiled<Real, 7, DOTS>(plan, l, st); break;
    case 8: launch_tiled<Real, 8, DOTS>(plan, l, st); break;
    case 9: launch_tiled<Real, 9, DOTS>(plan, l, st); break;
    case 10: launch_tiled<Real, 10, DOTS>(plan, l, st); break;
    case 11: launch_tiled<Real, 11, DOTS>(plan, l, st); break;
    case 12: launch_tiled<Real, 12, DOTS>(plan, l, st); break;
    default: throw Error{-2, "unsupported tile exponent"};
    }
}

void apply_launch(const ApplyPlan &plan, const ApplyLaunch &l, cudaStream_t st) {
    if (l.shards) {
        RP_REQUIRE(plan.rows.ok, -2,
                   "a sharded apply needs the row kernel: states of at least 2^19 complex64 or "
                   "2^18 complex128 elements, at most 2048 terms after splitting complex "
                   "coefficients");
        RP_REQUIRE(l.out && ((uintptr_t)l.out & 15) == 0, -2, "the output shard must be 16-byte aligned");
        RowLaunch r;
        r.out = l.out;
        r.alpha = l.alpha;
        r.alpha_dev = l.alpha_dev;
        r.accumulate = l.accumulate;
        r.active = l.active;
        r.err = l.err;
        r.tile0 = l.tile0;
        r.tile_count = l.tile_count;
        r.shards = l.shards;
        r.shard_bits = l.shard_bits;
        r.shard_rank = l.shard_rank;
        rows_launch(plan.rows, plan.len, plan.dtype, r, st);
        return;
    }
    RP_REQUIRE(l.in && l.out, -2, "null vector pointer");
    RP_REQUIRE(l.in != l.out, -2, "apply needs distinct input and output buffers");
    RP_REQUIRE(((uintptr_t)l.in & 15) == 0 && ((uintptr_t)l.out & 15) == 0, -2,
               "vectors must be 16-byte aligned");
    RP_REQUIRE(l.tile_count == 0 || plan.rows.ok, -2, "output tile ranges need the row kernel");
    if (plan.cfg.direct) {
        RP_REQUIRE(l.ndot == 0, -2, "fused projections need the tiled kernel");
        const uint32_t D = 1u << plan.len;
        const int threads = 32;
        const int blocks = (int)((D + threads - 1) / threads);
        if (plan.dtype == 2)
            k_apply_direct<double><<<blocks, threads, 0, st>>>(
                (const Cplx<double> *)l.in, (Cplx<double> *)l.out,
                (const DirectTerm<double> *)plan.d_direct, plan.nterms, D, l.alpha, l.alpha_dev,
                l.accumulate, l.active);
        else
            k_apply_direct<float><<<blocks, threads, 0, st>>>(
                (const Cplx<float> *)l.in, (Cplx<float> *)l.out,
                (const DirectTerm<float> *)plan.d_direct, plan.nterms, D, l.alpha, l.alpha_dev,
                l.accumulate, l.active);
        RP_CUDA(cudaGetLastError());
        return;
    }
    RP_REQUIRE(l.ndot <= MAX_FUSED_DOTS, -2, "too many fused projections");
    RP_REQUIRE(l.ndot == 0 || (l.dot_vecs && l.partials), -2, "fused projections need buffers");
    if (plan.ngroups == 0) {
        // no terms: H = 0
        const size_t bytes = ((size_t)1 << plan.len) * elem_size(plan.dtype);
        if (!l.accumulate) RP_CUDA(cudaMemsetAsync(l.out, 0, bytes, st));
        if (l.ndot) {
            const size_t pb = (size_t)apply_grid(plan) * l.ndot * 2 * sizeof(double);
            RP_CUDA(cudaMemsetAsync(l.partials, 0, pb, st));
        }
        return;
    }
    if (plan.rows.ok) {
        RowLaunch r;
        r.in = l.in;
        r.out = l.out;
        r.alpha = l.alpha;
        r.alpha_dev = l.alpha_dev;
        r.accumulate = l.accumulate;
        r.active = l.active;
        r.dot_vecs = l.dot_vecs;
        r.ndot = l.ndot;
        r.partials = l.partials;
        r.err = l.err;
        r.tile0 = l.tile0;
        r.tile_count = l.tile_count;
        rows_launch(plan.rows, plan.len, plan.dtype, r, st);
        return;
    }
    if (plan.dtype == 2) {
        if (l.ndot) dispatch_B<double, true>(plan, l, st);
        else dispatch_B<double, false>(plan, l, st);
    } else {
        if (l.ndot) dispatch_B<float, true>(plan, l, st);
        else dispatch_B<float, false>(plan, l, st);
    }
}

}  // namespace rp
