// Row-layout H.psi kernel for sm_100a (the default for large states).
//
// Each source tile (256 rows x 128 bytes = 32 KB: 4096 complex64 or 2048
// complex128 elements) is brought into shared memory by one 2-D TMA tensor
// copy with the 128-byte swizzle: the 16-byte chunk q of row r lands at chunk
// q ^ (r & 7).  Consumer thread t owns output row t.  For a term with in-tile
// X part xl = (xr, xq, x0) -- row XOR, chunk XOR, element-in-chunk XOR -- the
// source of output element (t, chunk p, e) is (t ^ xr, chunk p ^ xq, e ^ x0).
// The chunk XOR folds into the swizzle XOR of the shared-memory address, so
// the in-row permutation costs nothing; only the swap inside a 16-byte chunk
// (x0, FP32 only), its sign (z0) and the coefficient kind remain, as eight
// compile-time cases chosen by a warp-uniform switch.  The column-dependent
// sign is one select per chunk from a per-term 8-bit mask.  Output rows are
// written once.  Complex coefficients are split into a real and an imaginary
// term on the host, so every term costs two FMAs per element.
//
// Tile order: CTA c handles tiles c, c + grid, ...; the output tiles in
// flight form a block of `grid` consecutive tiles, whose source tiles for a
// group xh are that block XOR xh.  Groups are visited in increasing xh, so
// groups sharing the high bits of xh read overlapping source blocks back to
// back from L2.  Two CTAs per SM (2 x 148 = 296 CTAs) give 16 consumer warps
// per SM to hide shared-memory and FMA latency.
//
// Fused diagonal (DIAG variants, Hamiltonians with at least ROW_DIAG_MIN
// real Z strings): those terms leave the term list; with group 0 (the
// output's own tile) every row sums their coefficients, signed by its high
// index bits, into one bucket per in-row Z pattern, and a Walsh-Hadamard
// transform over the in-row bits gives each element's diagonal factor,
// applied once to the own row.
//
// Sharded variant (k_apply_rows_shard): one output shard of a state split by
// its top qubits, with one tensor map per input shard; each source tile is
// loaded from the shard holding it (this GPU's memory or a peer's), the Z
// signs use the global tile index.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "rp_apply.cuh"
#include "rp_apply_rows.cuh"
#include "rp_rows_dev.cuh"

namespace rp {

static int log2i(uint64_t v) {
    int l = 0;
    while ((1ull << l) < v) l++;
    return l;
}

void rowplan_build(RowPlan &rp, int len, int dtype, const uint64_t *bits, const double *coeff,
                   int64_t nterms, bool any_len, bool fuse_diag) {
    rp = RowPlan{};
    const int esz = dtype == 2 ? 16 : 8;
    const int C = 128 / esz;         // elements per row
    const int EPC = 16 / esz;        // elements per 16-byte chunk
    const int logC = log2i(C);
    const int logE = log2i(EPC);
    const int B = logC + 8;
    // fewer than 128 tiles: the first-generation kernel (unless the caller
    // only needs the table, as the batched kernel does: one tile suffices)
    if (len < (any_len ? B : B + 7)) return;
    struct T {
        uint32_t x, z;
        double c;
        int kind;
    };
    std::vector<T> ts;
    for (int64_t k = 0; k < nterms; k++) {
        uint32_t x = 0, z = 0;
        for (int i = 0; i < len; i++) {
            x |= (uint32_t)((bits[k] >> (2 * i)) & 1) << i;
            z |= (uint32_t)((bits[k] >> (2 * i + 1)) & 1) << i;
        }
        const double cr = coeff[2 * k], ci = coeff[2 * k + 1];
        if (cr != 0.0 || ci == 0.0) ts.push_back({x, z, cr, 0});
        if (ci != 0.0) ts.push_back({x, z, ci, 1});
    }
    if (fuse_diag) {
        const auto real_diag = [](const T &t) { return t.x == 0 && t.kind == 0; };
        const int nd = (int)std::count_if(ts.begin(), ts.end(), real_diag);
        if (nd >= ROW_DIAG_MIN) {
            std::vector<T> d;
            std::vector<T> rest;
            for (const T &t : ts) (real_diag(t) ? d : rest).push_back(t);
            ts.swap(rest);
            std::stable_sort(d.begin(), d.end(), [C](const T &a, const T &b) {
                return (a.z & (uint32_t)(C - 1)) < (b.z & (uint32_t)(C - 1));
            });
            rp.dstart.assign(C + 1, 0);
            for (const T &t : d) {
                rp.diag.push_back({t.z >> logC, (float)t.c, t.c});
                rp.dstart[(t.z & (uint32_t)(C - 1)) + 1]++;
            }
            for (int b = 0; b < C; b++) rp.dstart[b + 1] += rp.dstart[b];
            rp.ndiag = nd;
        }
    }
    if ((int)ts.size() > ROW_MAX_TERMS || rp.ndiag > ROW_MAX_TERMS) {
        rp = RowPlan{};
        return;
    }
    // by source tile (x >> B); in fused-diagonal (spin-chain) plans also by
    // the full X mask, so that terms reading the same source row with the
    // same case are adjacent and share one row load (ROW_SAME_SRC)
    const bool runs = rp.ndiag > 0;
    std::stable_sort(ts.begin(), ts.end(), [B, runs](const T &a, const T &b) {
        if ((a.x >> B) != (b.x >> B)) return (a.x >> B) < (b.x >> B);
        return runs && a.x < b.x;
    });
    for (size_t k = 0; k < ts.size(); k++) {
        const uint32_t xh = ts[k].x >> B;
        bool same = false;
        if (rp.groups.empty() || rp.groups.back().xh != xh)
            rp.groups.push_back({xh, (uint32_t)k, 0u, 0u});
        else
            same = runs && ts[k].x == ts[k - 1].x && ts[k].kind == ts[k - 1].kind &&
                   ((ts[k].z ^ ts[k - 1].z) & (uint32_t)(EPC - 1)) == 0;
        rp.groups.back().count++;
        const uint32_t xl = ts[k].x & ((1u << B) - 1);
        const uint32_t xr = xl >> logC, xc = xl & (uint32_t)(C - 1);
        const uint32_t xq = xc >> logE, x0 = xc & (uint32_t)(EPC - 1);
        const uint32_t zc = ts[k].z & (uint32_t)(C - 1);
        const uint32_t zq = zc >> logE, z0 = zc & (uint32_t)(EPC - 1);
        // chunk sign: bit p = parity(zq & (p ^ xq)) (source chunk p ^ xq)
        uint32_t jc = 0;
        for (int p = 0; p < 8; p++) jc |= (uint32_t)(__builtin_popcount(zq & (p ^ xq)) & 1) << p;
        RowTerm<float> r{};
        r.cs = xr | (xq << 8) | ((x0 | (z0 << 1) | ((uint32_t)ts[k].kind << 2)) << 11) |
               (same ? ROW_SAME_SRC : 0u);
        r.z = ts[k].z;
        r.js = jc;
        r.cf = (float)ts[k].c;
        r.cd = ts[k].c;
        rp.terms.push_back(r);
    }
    // the fused diagonal is applied with group 0, which must then be the
    // output's own tile (x >> B == 0), with or without terms of its own
    if (rp.ndiag && (rp.groups.empty() || rp.groups[0].xh != 0))
        rp.groups.insert(rp.groups.begin(), RowGroup{0u, 0u, 0u, 0u});
    if ((int)rp.groups.size() > ROW_MAX_GROUPS) {
        rp = RowPlan{};
        return;
    }
    rp.ok = true;
    rp.B = B;
    rp.logC = logC;
    rp.ntiles = 1 << (len - B);
    rp.nterms = (int)rp.terms.size();
    // CTAs in flight: two per SM by default (measured fastest on B200:
    // 47.7 ms vs 67.3 ms with one per SM and 77.6 ms with an aligned
    // 128-CTA window at N = 56); RPB200_ROW_GRID overrides it for tuning.
    int win = 2 * num_sms();
    if (const char *e = getenv("RPB200_ROW_GRID")) win = std::max(1, atoi(e));
    rp.window = std::min(rp.ntiles, win);
    const double D = std::ldexp(1.0, len);
    std::vector<uint32_t> hw;
    int lw = 0;
    while ((2 << lw) <= rp.window) lw++;
    for (auto &g : rp.groups) hw.push_back(g.xh >> lw);
    hw.erase(std::unique(hw.begin(), hw.end()), hw.end());
    rp.alg_bytes_smem = (double)(rp.groups.size() + 1) * D * esz;
    rp.alg_bytes_dram = (double)(hw.size() + 1) * D * esz;
}

void rowplan_upload(RowPlan &rp) {
    if (!rp.ok) return;
    rowplan_free(rp);
    RP_CUDA(cudaMalloc(&rp.d_terms, std::max<size_t>(16, rp.terms.size() * sizeof(RowTerm<float>))));
    RP_CUDA(cudaMemcpy(rp.d_terms, rp.terms.data(), rp.terms.size() * sizeof(RowTerm<float>),
                       cudaMemcpyHostToDevice));
    RP_CUDA(cudaMalloc((void **)&rp.d_groups, std::max<size_t>(16, rp.groups.size() * sizeof(RowGroup))));
    RP_CUDA(cudaMemcpy(rp.d_groups, rp.groups.data(), rp.groups.size() * sizeof(RowGroup),
                       cudaMemcpyHostToDevice));
    if (rp.ndiag) {
        RP_CUDA(cudaMalloc((void **)&rp.d_diag, rp.diag.size() * sizeof(RowDiag)));
        RP_CUDA(cudaMemcpy(rp.d_diag, rp.diag.data(), rp.diag.size() * sizeof(RowDiag),
                           cudaMemcpyHostToDevice));
        RP_CUDA(cudaMalloc((void **)&rp.d_dstart, rp.dstart.size() * sizeof(uint32_t)));
        RP_CUDA(cudaMemcpy(rp.d_dstart, rp.dstart.data(), rp.dstart.size() * sizeof(uint32_t),
                           cudaMemcpyHostToDevice));
    }
}

void rowplan_free(RowPlan &rp) {
    if (rp.d_terms) cudaFree(rp.d_terms);
    if (rp.d_groups) cudaFree(rp.d_groups);
    if (rp.d_diag) cudaFree(rp.d_diag);
    if (rp.d_dstart) cudaFree(rp.d_dstart);
    rp.d_terms = nullptr;
    rp.d_groups = nullptr;
    rp.d_diag = nullptr;
    rp.d_dstart = nullptr;
}

// ---------------------------------------------------------------------------
// Device code
// ---------------------------------------------------------------------------
template <typename Real>
struct RowArgs {
    Cplx<Real> *out;
    const RowTerm<float> *terms;
    const RowGroup *groups;
    int nterms, ngroups, ntiles, stages;
    uint32_t tile0;          // first output tile of this launch (ntiles from there)
    // sharded launch: output tiles are local tiles of shard gtile0 >> lbits;
    // source tile s (global) is local tile s & (2^lbits - 1) of map s >> lbits
    uint32_t gtile0;
    int lbits, nmaps;
    // fused diagonal (DIAG kernels): ndiag real Z strings by in-row bucket
    const RowDiag *diag;
    const uint32_t *dstart;
    int ndiag;
    double alpha;
    const double *alpha_dev;
    int accumulate;
    const int *active;
    const Cplx<Real> *const *dot_vecs;
    int ndot;
    double *partials;
    unsigned *err;
    // the failure-path test hook: CTA 0's producer withholds the tile copy of
    // iteration hold_it (-1: none), so that its consumers wait on a barrier
    // that never completes, and CTA 0's pipeline waits give up after
    // wait_polls polls (every other wait: WAIT_LIMIT)
    uint32_t wait_polls;
    long hold_it;
};

constexpr int ROW_P = 256;          // consumer threads = rows per tile
constexpr int ROW_NW = ROW_P / 32;
constexpr unsigned ROW_TILE_BYTES = 256 * 128;

// The fused diagonal of one output row (index bits above the in-row ones:
// hi), added to acc: bucket sums a_b = sum_{t: z_t & (C-1) = b} c_t
// (-1)^popc(zhi_t & hi), then a Walsh-Hadamard transform over the in-row
// bits gives d(e) = sum_b a_b (-1)^popc(b & e) for every element e, applied
// to the own row read from the staged tile at rq (no permutation).
template <typename Real>
__device__ __forceinline__ void apply_diag(Cplx<Real> (&acc)[128 / sizeof(Cplx<Real>)],
                                           const RowDiag *sdiag, const uint32_t *sdstart, uint32_t hi,
                                           uint32_t rq) {
    constexpr int C = 128 / (int)sizeof(Cplx<Real>);
    Real d[C];
#pragma unroll
    for (int b = 0; b < C; b++) {
        Real sum = Real(0);
        const uint32_t t1 = sdstart[b + 1];
        for (uint32_t t = sdstart[b]; t < t1; t++) {
            const RowDiag dt = sdiag[t];
            Real c;
            if constexpr (sizeof(Real) == 4) c = dt.cf;
            else c = dt.cd;
            sum += (__popc(dt.zhi & hi) & 1) ? -c : c;
        }
        d[b] = sum;
    }
#pragma unroll
    for (int h = 1; h < C; h <<= 1) {
#pragma unroll
        for (int e = 0; e < C; e++) {
            if (!(e & h)) {
                const Real u = d[e], v = d[e | h];
                d[e] = u + v;
                d[e | h] = u - v;
            }
        }
    }
    float4 w[8];
    load_row(w, rq);
#pragma unroll
    for (int p = 0; p < 8; p++) {
        if constexpr (C == 16) {
            acc[2 * p].x = fma(d[2 * p], w[p].x, acc[2 * p].x);
            acc[2 * p].y = fma(d[2 * p], w[p].y, acc[2 * p].y);
            acc[2 * p + 1].x = fma(d[2 * p + 1], w[p].z, acc[2 * p + 1].x);
            acc[2 * p + 1].y = fma(d[2 * p + 1], w[p].w, acc[2 * p + 1].y);
        } else {
            const double vx = __hiloint2double(__float_as_int(w[p].y), __float_as_int(w[p].x));
            const double vy = __hiloint2double(__float_as_int(w[p].w), __float_as_int(w[p].z));
            acc[p].x = fma(d[p], vx, acc[p].x);
            acc[p].y = fma(d[p], vy, acc[p].y);
        }
    }
}

// The row kernel's body.  maps points at kernel-parameter tensor maps: one
// over the whole input state, or (SHARD) one per input shard, a shard being
// this GPU's memory or a peer's.
template <typename Real, bool SHARD, bool DIAG>
__device__ __forceinline__ void apply_rows_body(const CUtensorMap *maps, const RowArgs<Real> a) {
    constexpr int C = 128 / (int)sizeof(Cplx<Real>);   // elements per row
    constexpr int LOGC = C == 16 ? 4 : 3;
    constexpr int B = LOGC + 8;
    extern __shared__ unsigned char smem_raw[];
    // 1024-byte alignment for the 128-byte swizzle pattern
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int S = a.stages;
    unsigned char *stage = smem;
    RowTerm<float> *sterms = reinterpret_cast<RowTerm<float> *>(smem + (size_t)S * ROW_TILE_BYTES);
    RowGroup *sgroups = reinterpret_cast<RowGroup *>(sterms + a.nterms);
    RowDiag *sdiag = reinterpret_cast<RowDiag *>(sgroups + a.ngroups);
    uint32_t *sdstart = reinterpret_cast<uint32_t *>(sdiag + (DIAG ? a.ndiag : 0));
    uint64_t *full = reinterpret_cast<uint64_t *>(sdstart + (DIAG ? (C + 4) & ~3 : 0));
    uint64_t *empty = full + S;
    double *red = reinterpret_cast<double *>(empty + S);
    __shared__ int s_abort;
    __shared__ long s_issued;

    if (a.active && *a.active == 0) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < a.nterms; i += blockDim.x) sterms[i] = a.terms[i];
    for (int i = tid; i < a.ngroups; i += blockDim.x) sgroups[i] = a.groups[i];
    if constexpr (DIAG) {
        for (int i = tid; i < a.ndiag; i += blockDim.x) sdiag[i] = a.diag[i];
        for (int i = tid; i <= C; i += blockDim.x) sdstart[i] = a.dstart[i];
    }
    if (a.ndot)
        for (int i = tid; i < ROW_NW * a.ndot * 4; i += blockDim.x) red[i] = 0.0;
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], ROW_NW);
        }
        s_abort = 0;
        s_issued = 0;
        fence_barrier_init();
    }
    __syncthreads();

    const int ntile_iters =
        (int)blockIdx.x < a.ntiles ? (a.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const long total = (long)ntile_iters * a.ngroups;
    const uint32_t polls = blockIdx.x == 0 ? a.wait_polls : WAIT_LIMIT;

    if (warp == ROW_NW) {
        if (lane == 0) {
            for (int i = 0; i < (SHARD ? a.nmaps : 1); i++)
                asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps[i]))
                             : "memory");
            long it = 0;
            for (; it < total; ++it) {
                const int s = (int)(it % S);
                const unsigned round = (unsigned)(it / S);
                if (!mbar_wait_bounded(&empty[s], (round & 1u) ^ 1u, a.err, polls)) {
                    atomicExch(&s_abort, 1);
                    break;
                }
                const long ti = it / a.ngroups;
                const int g = (int)(it - ti * a.ngroups);
                const uint32_t o = a.tile0 + blockIdx.x + (uint32_t)ti * gridDim.x;
                if (it == a.hold_it && blockIdx.x == 0) continue;   // test hook: never arrives
                mbar_arrive_expect_tx(&full[s], ROW_TILE_BYTES);
                if constexpr (SHARD) {
                    const uint32_t src = (a.gtile0 + o) ^ sgroups[g].xh;
                    const uint32_t lsrc = src & ((1u << a.lbits) - 1u);
                    tma_load_2d(stage + (size_t)s * ROW_TILE_BYTES, &maps[src >> a.lbits], 0,
                                (int)(lsrc * 256u), &full[s]);
                } else {
                    const uint32_t src = o ^ sgroups[g].xh;
                    tma_load_2d(stage + (size_t)s * ROW_TILE_BYTES, maps, 0, (int)(src * 256u), &full[s]);
                }
            }
            s_issued = it;
        }
    } else {
        const uint32_t row = (uint32_t)tid;
        const double scale = a.alpha * (a.alpha_dev ? *a.alpha_dev : 1.0);
        long it = 0;
        bool ok = true;
        for (int ti = 0; ti < ntile_iters && ok; ++ti) {
            const uint32_t o = a.tile0 + blockIdx.x + (uint32_t)ti * gridDim.x;
            const uint32_t og = SHARD ? a.gtile0 + o : o;   // global tile: the Z signs
            Cplx<Real> acc[C];
#pragma unroll
            for (int u = 0; u < C; u++) acc[u].x = acc[u].y = Real(0);
            for (int g = 0; g < a.ngroups; ++g, ++it) {
                const int s = (int)(it % S);
                const unsigned round = (unsigned)(it / S);
                const RowGroup gd = sgroups[g];
                const uint32_t src_hi = (og ^ gd.xh) << B;
                if (!mbar_wait_bounded(&full[s], round & 1u, a.err, polls)) {
                    ok = false;
                    break;
                }
                const uint32_t tile = smem_u32(stage + (size_t)s * ROW_TILE_BYTES);
                if constexpr (DIAG) {
                    // spin-chain plans: consecutive terms with the same X mask
                    // and case (ROW_SAME_SRC) share one load of their source row
                    auto decode = [&](uint32_t k, uint32_t &cs, uint32_t &jc, Real &c0) {
                        const uint4 d0 = *reinterpret_cast<const uint4 *>(&sterms[k]);
                        cs = d0.x;
                        jc = d0.z;
                        const uint32_t sr = row ^ (cs & 0xFFu);
                        const uint32_t s0 = (uint32_t)(__popc(d0.y & (src_hi | (sr << LOGC))) & 1);
                        if constexpr (sizeof(Real) == 4) c0 = __uint_as_float(d0.w);
                        else c0 = sterms[k].cd;
                        if (s0) c0 = -c0;
                    };
                    const uint32_t kend = gd.first + gd.count;
                    for (uint32_t k = gd.first; k < kend; ++k) {
                        uint32_t cs, jc;
                        Real c0;
                        decode(k, cs, jc, c0);
                        const uint32_t sr = row ^ (cs & 0xFFu);
                        const uint32_t xq = (cs >> 8) & 7u;
                        float4 w[8];
                        load_row(w, (tile + sr * 128u) | ((xq ^ (sr & 7u)) << 4));
                        switch ((cs >> 11) & 7u) {
#define RP_ROW_RUN(K)                                                          \
    case K:                                                                    \
        for (;;) {                                                             \
            row_case<Real, K>(acc, w, c0, jc);                                 \
            if (k + 1 >= kend || !(sterms[k + 1].cs & ROW_SAME_SRC)) break;    \
            ++k;                                                               \
            decode(k, cs, jc, c0);                                             \
        }                                                                      \
        break;
                            RP_ROW_RUN(0)
                            RP_ROW_RUN(1)
                            RP_ROW_RUN(2)
                            RP_ROW_RUN(3)
                            RP_ROW_RUN(4)
                            RP_ROW_RUN(5)
                            RP_ROW_RUN(6)
                            RP_ROW_RUN(7)
#undef RP_ROW_RUN
                        }
                    }
                } else {
                    for (uint32_t k = gd.first; k < gd.first + gd.count; ++k) {
                        const uint4 d0 = *reinterpret_cast<const uint4 *>(&sterms[k]);
                        const uint32_t cs = d0.x, z = d0.y, jc = d0.z;
                        const uint32_t sr = row ^ (cs & 0xFFu);
                        const uint32_t xq = (cs >> 8) & 7u;
                        const uint32_t s0 = (uint32_t)(__popc(z & (src_hi | (sr << LOGC))) & 1);
                        Real c0;
                        if constexpr (sizeof(Real) == 4) c0 = __uint_as_float(d0.w);
                        else c0 = sterms[k].cd;
                        if (s0) c0 = -c0;
                        // chunk p of the permuted source row sits at physical
                        // chunk p ^ xq ^ (sr & 7) of row sr
                        const uint32_t rq = (tile + sr * 128u) | ((xq ^ (sr & 7u)) << 4);
                        switch ((cs >> 11) & 7u) {
                            case 0: chunk_case<Real, 0>(acc, rq, c0, jc); break;
                            case 1: chunk_case<Real, 1>(acc, rq, c0, jc); break;
                            case 2: chunk_case<Real, 2>(acc, rq, c0, jc); break;
                            case 3: chunk_case<Real, 3>(acc, rq, c0, jc); break;
                            case 4: chunk_case<Real, 4>(acc, rq, c0, jc); break;
                            case 5: chunk_case<Real, 5>(acc, rq, c0, jc); break;
                            case 6: chunk_case<Real, 6>(acc, rq, c0, jc); break;
                            default: chunk_case<Real, 7>(acc, rq, c0, jc); break;
                        }
                    }
                }
                if constexpr (DIAG) {
                    // group 0 is the output's own tile: the diagonal factor
                    // d(u) = sum_t c_t (-1)^popc(z_t & u) times the own row
                    if (g == 0) apply_diag<Real>(acc, sdiag, sdstart, (og << 8) | row,
                                                 (tile + row * 128u) | ((row & 7u) << 4));
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[s]);
            }
            if (!ok) break;
            // write the row: C contiguous elements = 8 x 16 bytes
            Cplx<Real> *orow = a.out + ((size_t)o << B) + (size_t)row * C;
#pragma unroll
            for (int u = 0; u < C; u++) {
                Cplx<Real> r;
                r.x = (Real)(scale * (double)acc[u].x);
                r.y = (Real)(scale * (double)acc[u].y);
                acc[u] = r;
            }
            if (a.accumulate) {
#pragma unroll
                for (int u = 0; u < C; u++) {
                    const Cplx<Real> old = orow[u];
                    acc[u].x += old.x;
                    acc[u].y += old.y;
                }
            }
#pragma unroll
            for (int p = 0; p < 8; p++) {
                float4 q;
                if constexpr (sizeof(Real) == 4) {
                    q = make_float4(acc[2 * p].x, acc[2 * p].y, acc[2 * p + 1].x, acc[2 * p + 1].y);
                } else {
                    q = make_float4(__int_as_float(__double2loint(acc[p].x)),
                                    __int_as_float(__double2hiint(acc[p].x)),
                                    __int_as_float(__double2loint(acc[p].y)),
                                    __int_as_float(__double2hiint(acc[p].y)));
                }
                reinterpret_cast<float4 *>(orow)[p] = q;
            }
            if (a.ndot) {
                for (int i = 0; i < a.ndot; i++) {
                    const Cplx<Real> *u = a.dot_vecs[i] + ((size_t)o << B) + (size_t)row * C;
                    double sr = 0.0, si = 0.0;
#pragma unroll
                    for (int e = 0; e < C; e++) {
                        const Cplx<Real> uv = u[e];
                        sr = fma((double)uv.x, (double)acc[e].x, fma((double)uv.y, (double)acc[e].y, sr));
                        si = fma((double)uv.x, (double)acc[e].y, fma(-(double)uv.y, (double)acc[e].x, si));
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
        // let the copies still in flight land before the CTA exits (the
        // withheld test copy was never issued)
        if (tid == 0) {
            const long issued = s_issued;
            for (long it = issued - S; it < issued; ++it) {
                if (it < 0 || (it == a.hold_it && blockIdx.x == 0)) continue;
                mbar_wait_bounded(&full[it % S], (unsigned)((it / S) & 1), a.err);
            }
        }
        return;
    }
    if (a.ndot) {
        for (int i = tid; i < a.ndot; i += blockDim.x) {
            CompSum re, im;
            for (int w = 0; w < ROW_NW; w++) {
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

template <typename Real, int MINB, bool DIAG>
__global__ void __launch_bounds__(ROW_P + 32, MINB)
    k_apply_rows(const __grid_constant__ CUtensorMap tmap, const RowArgs<Real> a) {
    apply_rows_body<Real, false, DIAG>(&tmap, a);
}

// One output shard of a state split by its top qubits: the source tiles come
// from the shard that holds them (plain TMA loads, over NVLink for a peer's
// memory; no multicast).
struct RowShardMaps {
    CUtensorMap m[ROW_MAX_SHARDS];
};

template <typename Real, int MINB, bool DIAG>
__global__ void __launch_bounds__(ROW_P + 32, MINB)
    k_apply_rows_shard(const __grid_constant__ RowShardMaps maps, const RowArgs<Real> a) {
    apply_rows_body<Real, true, DIAG>(maps.m, a);
}

// ---------------------------------------------------------------------------
// Host launch
// ---------------------------------------------------------------------------
static int ilog2(uint32_t v) {
    int r = 0;
    while ((2u << r) <= v) r++;
    return r;
}

static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        RP_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        RP_REQUIRE(q == cudaDriverEntryPointSuccess && p, -3, "cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// The state viewed as rows of 128 bytes: inner dimension 32 floats (or 16
// doubles), outer dimension D / C rows; box = one 256-row tile, 128B swizzle.
CUtensorMap make_row_map(const void *base, int len, int dtype) {
    CUtensorMap m;
    const int esz = dtype == 2 ? 16 : 8;
    const int C = 128 / esz;
    const cuuint64_t inner = dtype == 2 ? 16 : 32;
    const cuuint64_t dims[2] = {inner, (cuuint64_t)((1ull << len) / C)};
    const cuuint64_t strides[1] = {128};
    const cuuint32_t box[2] = {(cuuint32_t)inner, 256};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = get_encode()(
        &m, dtype == 2 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
        const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    RP_REQUIRE(r == CUDA_SUCCESS, -3, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

// The failure-path test hook (rows_test_withhold): armed for one launch.
struct HoldTest {
    bool armed = false;
    long iteration = -1;
    uint32_t polls = WAIT_LIMIT;
};
static HoldTest g_hold;

void rows_test_withhold(long iteration, uint32_t polls) {
    RP_REQUIRE(iteration >= 0, -2, "the withheld iteration must be non-negative");
    RP_REQUIRE(polls >= 1024 && polls <= WAIT_LIMIT, -2,
               "wait_polls must be in [1024, " + std::to_string(WAIT_LIMIT) + "]");
    g_hold.armed = true;
    g_hold.iteration = iteration;
    g_hold.polls = polls;
}

template <typename Real>
static void launch_rows_t(const RowPlan &rp, int len, int dtype, const RowLaunch &l,
                          cudaStream_t st) {
    const bool diag = rp.ndiag > 0;
    const int C = 128 / (int)sizeof(Cplx<Real>);
    const size_t fixed = (size_t)rp.nterms * sizeof(RowTerm<float>) +
                         (size_t)rp.groups.size() * sizeof(RowGroup) +
                         (diag ? (size_t)rp.ndiag * sizeof(RowDiag) + (size_t)((C + 4) & ~3) * 4 : 0) +
                         (size_t)ROW_NW * l.ndot * 4 * sizeof(double) + 1024;
    // CTAs per SM (RPB200_ROW_CTAS, 1 or 2; default 2): the shared memory of
    // an SM (228 KB, 1 KB of it reserved per CTA) is split between them
    static int ctas = 0;
    if (!ctas) {
        const char *e = getenv("RPB200_ROW_CTAS");
        ctas = (e && atoi(e) == 1) ? 1 : 2;
    }
    const size_t budget = (ctas == 2 ? 113 * 1024 : 227 * 1024) - 64;
    int S = (int)std::min<size_t>(6, (budget - fixed - 16 * 8) / (ROW_TILE_BYTES + 16));
    RP_REQUIRE(S >= 2, -2, "Hamiltonian table too large for the row kernel");
    const size_t smem = (size_t)S * ROW_TILE_BYTES + fixed + (size_t)2 * S * sizeof(uint64_t);
    const bool shard = l.shards != nullptr;
    auto kern = ctas == 2 ? (diag ? k_apply_rows<Real, 2, true> : k_apply_rows<Real, 2, false>)
                          : (diag ? k_apply_rows<Real, 1, true> : k_apply_rows<Real, 1, false>);
    auto kern_sh = ctas == 2 ? (diag ? k_apply_rows_shard<Real, 2, true> : k_apply_rows_shard<Real, 2, false>)
                             : (diag ? k_apply_rows_shard<Real, 1, true> : k_apply_rows_shard<Real, 1, false>);
    static size_t attr[2][2][2] = {};
    if (smem > attr[shard][diag][ctas - 1]) {
        if (shard)
            RP_CUDA(cudaFuncSetAttribute(kern_sh, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        else
            RP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr[shard][diag][ctas - 1] = smem;
    }
    const int lbits = shard ? ilog2((uint32_t)rp.ntiles) - l.shard_bits : 0;
    const int local_tiles = shard ? rp.ntiles >> l.shard_bits : rp.ntiles;
    RowArgs<Real> a;
    a.out = static_cast<Cplx<Real> *>(l.out);
    a.terms = static_cast<const RowTerm<float> *>(rp.d_terms);
    a.groups = rp.d_groups;
    a.nterms = rp.nterms;
    a.ngroups = (int)rp.groups.size();
    a.ntiles = l.tile_count ? (int)l.tile_count : local_tiles;
    a.tile0 = l.tile0;
    a.gtile0 = shard ? (uint32_t)l.shard_rank << lbits : 0u;
    a.lbits = lbits;
    a.nmaps = shard ? 1 << l.shard_bits : 1;
    a.diag = rp.d_diag;
    a.dstart = rp.d_dstart;
    a.ndiag = rp.ndiag;
    a.stages = S;
    a.alpha = l.alpha;
    a.alpha_dev = l.alpha_dev;
    a.accumulate = l.accumulate;
    a.active = l.active;
    a.dot_vecs = reinterpret_cast<const Cplx<Real> *const *>(l.dot_vecs);
    a.ndot = l.ndot;
    a.partials = l.partials;
    a.err = l.err;
    a.wait_polls = WAIT_LIMIT;
    a.hold_it = -1;
    if (g_hold.armed) {
        a.wait_polls = g_hold.polls;
        a.hold_it = g_hold.iteration;
        g_hold = HoldTest{};
    }
    if (shard) {
        RowShardMaps maps;
        std::memset(&maps, 0, sizeof(maps));
        for (int i = 0; i < a.nmaps; i++) maps.m[i] = make_row_map(l.shards[i], len - l.shard_bits, dtype);
        kern_sh<<<std::min(rp.window, local_tiles), ROW_P + 32, smem, st>>>(maps, a);
    } else {
        const CUtensorMap map = make_row_map(l.in, len, dtype);
        kern<<<rp.window, ROW_P + 32, smem, st>>>(map, a);
    }
    RP_CUDA(cudaGetLastError());
}

void rows_launch(const RowPlan &rp, int len, int dtype, const RowLaunch &l, cudaStream_t st) {
    RP_REQUIRE(rp.ok, -2, "row kernel not planned for this Hamiltonian");
    RP_REQUIRE(l.ndot <= 64, -2, "too many fused projections");
    if (l.shards) {
        RP_REQUIRE(l.shard_bits >= 1 && l.shard_bits <= ilog2(ROW_MAX_SHARDS), -2,
                   "a sharded apply takes 2 to " + std::to_string(ROW_MAX_SHARDS) + " shards");
        RP_REQUIRE(rp.ntiles >= (1 << l.shard_bits), -2,
                   "every shard must hold at least one row tile (2^" + std::to_string(rp.B) + " elements)");
        RP_REQUIRE(l.shard_rank >= 0 && l.shard_rank < (1 << l.shard_bits), -2, "shard index out of range");
        RP_REQUIRE(l.ndot == 0, -2, "fused projections are not taken in a sharded apply");
        for (int i = 0; i < (1 << l.shard_bits); i++) {
            RP_REQUIRE(l.shards[i] && ((uintptr_t)l.shards[i] & 15) == 0, -2,
                       "shard pointers must be non-null and 16-byte aligned");
            RP_REQUIRE(l.shards[i] != l.out, -2, "the output may not be an input shard");
        }
    }
    const uint64_t out_tiles = l.shards ? (uint64_t)rp.ntiles >> l.shard_bits : (uint64_t)rp.ntiles;
    RP_REQUIRE((uint64_t)l.tile0 + l.tile_count <= out_tiles, -2, "output tile range out of bounds");
    RP_REQUIRE(l.tile_count == 0 || l.ndot == 0, -2, "fused projections need the whole output");
    RP_REQUIRE(l.tile_count != 0 || l.tile0 == 0, -2, "a tile offset needs a tile count");
    if (dtype == 2) launch_rows_t<double>(rp, len, dtype, l, st);
    else launch_rows_t<float>(rp, len, dtype, l, st);
}

}  // namespace rp
