// Restarted Krylov exp(-(beta + i t) H) psi (Eiermann-Ernst), GPU-resident.
//
// Control flow follows Krylov::evolve / arnoldi / orthogonalize of the
// reference (inc/algo.h:77-173, 267-365) step for step -- the same pass
// criterion (eta = 1/sqrt 2, at most three passes, first comparison against
// eta/2), the same breakdown rule, the same growing block Hessenberg matrix
// and the same convergence test on ||Hexp0|| -- so the number of H.psi
// products and restarts match the reference.  What differs is how each step
// touches HBM:
//   * projections of a pass are taken all at once (classical Gram-Schmidt
//     per pass; the first pass's projections are fused into the H.psi
//     epilogue) instead of one inner product + axpy per basis vector;
//   * the update w -= sum h_i v_i and ||w|| are one fused pass;
//   * the basis is stored unnormalised with per-vector scale factors, so no
//     normalisation pass is made;
//   * all decisions run in tiny device kernels gated by device flags, so a
//     whole Arnoldi cycle is enqueued without a host round trip, and the host
//     synchronises once per restart.
// Inner products, norms, H, Hfull and its exponential are FP64 on the GPU for
// both vector precisions.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "rp_expm_impl.cuh"
#include "rp_krylov.cuh"

namespace rp {

static size_t esize(int dtype) { return dtype == 2 ? 16 : 8; }

// The first orthogonalisation pass's projections <v_i|w> can be taken in the
// H.psi kernel's epilogue (w never leaves the SM before it is projected) or by
// the grouped projection kernel after the apply.  The separate kernel streams
// the basis at a higher fraction of HBM bandwidth than the epilogue, whose
// per-row warp reductions slow the apply, so it is the default;
// RPB200_FUSED_DOTS=1 selects the fused form.
static bool fused_projections() {
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("RPB200_FUSED_DOTS");
        v = (e && e[0] == '1') ? 1 : 0;
    }
    return v == 1;
}

static void grow_hfull(KryWorkspace &ws, int need, cudaStream_t st) {
    if (need <= ws.hcap) return;
    int cap = std::max(ws.hcap ? ws.hcap : 4 * ws.krydim, 32);
    while (cap < need) cap *= 2;
    void *nh = nullptr, *ns = nullptr;
    RP_CUDA(cudaMalloc(&nh, (size_t)cap * cap * sizeof(cd)));
    RP_CUDA(cudaMemsetAsync(nh, 0, (size_t)cap * cap * sizeof(cd), st));
    if (ws.hfull) {
        RP_CUDA(cudaMemcpy2DAsync(nh, (size_t)cap * sizeof(cd), ws.hfull,
                                  (size_t)ws.hcap * sizeof(cd), (size_t)ws.hcap * sizeof(cd),
                                  ws.hcap, cudaMemcpyDeviceToDevice, st));
        RP_CUDA(cudaStreamSynchronize(st));
        cudaFree(ws.hfull);
    }
    RP_CUDA(cudaMalloc(&ns, ((size_t)2 * cap * cap + expm_scratch_elems(cap)) * sizeof(cd)));
    if (ws.escratch) cudaFree(ws.escratch);
    ws.hfull = nh;
    ws.escratch = ns;
    ws.hcap = cap;
}

void workspace_release(KryWorkspace &ws) {
    for (void *p : ws.u) cudaFree(p);
    ws.u.clear();
    if (ws.y) cudaFree(ws.y);
    if (ws.dev) cudaFree(ws.dev);
    if (ws.partials) cudaFree(ws.partials);
    if (ws.norm_partials) cudaFree(ws.norm_partials);
    if (ws.hfull) cudaFree(ws.hfull);
    if (ws.escratch) cudaFree(ws.escratch);
    if (ws.err) cudaFree(ws.err);
    if (ws.tab) cudaFree(ws.tab);
    ws = KryWorkspace{};
}

void workspace_ensure(KryWorkspace &ws, int len, int dtype, int krydim) {
    if (ws.dev && ws.len == len && ws.dtype == dtype) {
        if (krydim <= ws.krydim) return;
        // a larger basis for the same state: add vectors, keep the rest
        const size_t vb = ws.D * esize(dtype);
        while (ws.krydim < krydim) {
            void *p = nullptr;
            if (cudaMalloc(&p, vb) != cudaSuccess) {
                cudaGetLastError();
                throw Error{-4, "device out of memory for the Krylov workspace"};
            }
            ws.u.push_back(p);
            ws.krydim++;
        }
        return;
    }
    workspace_release(ws);
    ws.len = len;
    ws.dtype = dtype;
    ws.krydim = krydim;
    ws.D = 1ull << len;
    const size_t vb = ws.D * esize(dtype);
    try {
        ws.u.resize(krydim + 1, nullptr);
        for (int i = 0; i <= krydim; i++) RP_CUDA(cudaMalloc(&ws.u[i], vb));
        RP_CUDA(cudaMalloc(&ws.y, vb));
        RP_CUDA(cudaMalloc((void **)&ws.dev, sizeof(KryDev)));
        const int g = std::max(num_sms(), reduce_grid());
        RP_CUDA(cudaMalloc((void **)&ws.partials, (size_t)g * (MAX_KRYLOV + 1) * 2 * sizeof(double)));
        RP_CUDA(cudaMalloc((void **)&ws.norm_partials, (size_t)g * sizeof(double)));
        RP_CUDA(cudaMalloc((void **)&ws.err, sizeof(unsigned)));
        RP_CUDA(cudaMemset(ws.err, 0, sizeof(unsigned)));
        RP_CUDA(cudaMalloc((void **)&ws.tab, (MAX_KRYLOV + 1) * sizeof(void *)));
    } catch (Error &e) {
        workspace_release(ws);
        throw Error{-4, "device out of memory for the Krylov workspace (" + e.msg + ")"};
    }
}

// ---------------------------------------------------------------------------
// Control kernels (one CTA each; they only touch the small state)
// ---------------------------------------------------------------------------
__global__ void k_kry_init(KryDev *s, double beta0) {
    if (threadIdx.x == 0) {
        memset(s, 0, offsetof(KryDev, sigma));
        s->beta0 = beta0;
        s->sigma[0] = 1.0 / beta0;
    }
}

__global__ void k_kry_begin(KryDev *s, int krydim, int restart) {
    if (threadIdx.x == 0) {
        s->active = 1;
        s->again = 0;
        s->m_eff = krydim;
        s->brokedown = 0;
        if (restart) {
            // the last basis vector v_m is the next starting vector
            s->sigma[0] = s->sigma[krydim];
            s->oldbeta = s->beta;
        }
    }
    for (int i = threadIdx.x; i < 2 * krydim * krydim; i += blockDim.x) s->H[i] = 0.0;
}

// h_i = sigma_i <u_i|w> for i <= j, reduced in a fixed order from per-CTA
// partials, one warp per basis vector.
__global__ void k_kry_proj(KryDev *s, const double *partials, int grid, int j, int pass) {
    if (!s->active) return;
    if (pass > 1 && !s->again) return;
    const int n = j + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = warp; i < n; i += nw) {
        const double re = warp_compsum(partials + (size_t)i * 2, grid, (size_t)n * 2);
        const double im = warp_compsum(partials + (size_t)i * 2 + 1, grid, (size_t)n * 2);
        if (lane != 0) continue;
        const double sg = s->sigma[i];
        const double hr = sg * re, hi = sg * im;
        if (pass == 1) {
            s->hacc[2 * i] = hr;
            s->hacc[2 * i + 1] = hi;
        } else {
            s->hacc[2 * i] += hr;
            s->hacc[2 * i + 1] += hi;
        }
        // w -= h_i v_i = (h_i sigma_i) u_i
        s->coef[2 * i] = -hr * sg;
        s->coef[2 * i + 1] = -hi * sg;
    }
}

// ||w|| after a pass and the pass criterion of Krylov::orthogonalize
// (inc/algo.h:86-106): continue while niter < 3, norm != 0 and
// norm < eta * old_norm, old_norm starting at eta / 2.
__global__ void k_kry_norm(KryDev *s, const double *np, int grid, int j, int krydim, int pass) {
    if (!s->active) return;
    if (pass > 1 && !s->again) return;
    const double sq = warp_compsum(np, grid, 1);   // one warp
    if (threadIdx.x != 0) return;
    const double norm = sqrt(sq);
    const double eta = 1.0 / sqrt(2.0);
    const double old = pass == 1 ? eta / 2 : s->norm;
    s->old_norm = old;
    s->norm = norm;
    s->niter = pass;
    const bool again = pass < 3 && norm != 0.0 && norm < eta * old;
    s->again = again;
    if (again) return;
    s->passes += pass;
    s->prods += pass * (j + 2);
    const bool ok = norm != 0.0 && norm >= eta * old;
    s->beta = norm;
    for (int i = 0; i <= j; i++) {
        s->H[2 * (i + j * krydim)] = s->hacc[2 * i];
        s->H[2 * (i + j * krydim) + 1] = s->hacc[2 * i + 1];
    }
    if (ok) {
        if (j != krydim - 1) {
            s->H[2 * ((j + 1) + j * krydim)] = norm;
            s->H[2 * ((j + 1) + j * krydim) + 1] = 0.0;
        }
        s->sigma[j + 1] = 1.0 / norm;
    } else {
        s->m_eff = j + 1;
        s->brokedown = 1;
        s->active = 0;
    }
}

// Grow Hfull by the cycle's block (Algorithm 2 of Eiermann & Ernst, as in
// inc/algo.h:303-328), exponentiate f * Hfull (f = -(t_imag + i t_real)),
// take the last m entries of column 0 (Hexp0), its norm, and the update
// coefficients beta0 * Hexp0_i * sigma_i.
__global__ void __launch_bounds__(512) k_kry_expm(KryDev *s, cd *hfull, int hcap, cd *scratch,
                                                  int krydim, int cycle, double fr, double fi) {
    extern __shared__ double smem[];
    const int m = s->m_eff;
    const int base = (cycle - 1) * krydim;
    const int n = base + m;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e % n, j = e / n;
        if (i >= base || j >= base) hfull[i + (size_t)j * hcap] = cd{0.0, 0.0};
    }
    __syncthreads();
    if (threadIdx.x == 0 && cycle > 1) hfull[base + (size_t)(base - 1) * hcap] = cd{s->oldbeta, 0.0};
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
        const int i = e % m, j = e / m;
        hfull[(base + i) + (size_t)(base + j) * hcap] =
            cd{s->H[2 * (i + j * krydim)], s->H[2 * (i + j * krydim) + 1]};
    }
    __syncthreads();
    cd *A = scratch, *E = scratch + (size_t)n * n, *ws = E + (size_t)n * n;
    const cd f{fr, fi};
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e % n, j = e / n;
        A[e] = cmul(f, hfull[i + (size_t)j * hcap]);
    }
    __syncthreads();
    expm_block(n, A, E, ws, smem);
    if (threadIdx.x == 0) {
        double sq = 0.0;
        for (int i = 0; i < m; i++) {
            const cd e = E[base + i];
            sq += e.x * e.x + e.y * e.y;
        }
        s->nrm = sqrt(sq);
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const cd e = E[base + i];
        const double c = s->beta0 * s->sigma[i];
        s->ycoef[2 * i] = c * e.x;
        s->ycoef[2 * i + 1] = c * e.y;
    }
}

double vec_norm_sync(int dtype, uint64_t n, const void *v, KryWorkspace *ws, cudaStream_t st) {
    const int g = reduce_grid();
    double *part = ws && ws->partials ? ws->partials : nullptr;
    if (!part) part = static_cast<double *>(scratch_get(SCR_NORM, (size_t)g * 2 * sizeof(double), st));
    VecTable tab{};
    tab.p[0] = v;
    multi_dot_partials(dtype, n, tab, 1, v, part, nullptr, nullptr, st);
    std::vector<double> h((size_t)g * 2);
    RP_CUDA(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
    double hi = 0.0, lo = 0.0;
    for (int i = 0; i < g; i++) {
        double x = h[2 * i];
        double s = hi + x, bb = s - hi;
        lo += (hi - (s - bb)) + (x - bb);
        hi = s;
    }
    return std::sqrt(hi + lo);
}

struct KryHeader {
    int active, again, niter, m_eff, brokedown, passes, prods, pad;
    double norm, old_norm, beta, oldbeta, beta0, nrm;
};
static_assert(sizeof(KryHeader) == offsetof(KryDev, sigma), "header layout");

void krylov_evolve(const ApplyPlan &plan, KryWorkspace &ws, void *psi, double t_real,
                   double t_imag, int krydim, double tol, int max_iters, EvolveStats *stats,
                   cudaStream_t st) {
    RP_REQUIRE(krydim >= 2 && krydim <= MAX_KRYLOV, -2, "krydim must be in [2, 64]");
    RP_REQUIRE(psi, -2, "null state vector");
    EvolveStats S{};
    if (stats) *stats = S;
    // State::evolve returns immediately for t == 0 and beta == 0 (inc/state.h:418)
    if (t_real == 0.0 && t_imag == 0.0) return;
    workspace_ensure(ws, plan.len, plan.dtype, krydim);
    const uint64_t D = ws.D;
    const int dtype = plan.dtype;
    const double beta0 = vec_norm_sync(dtype, D, psi, &ws, st);
    if (beta0 == 0.0) return;   // exp(A) 0 = 0
    RP_CUDA(cudaMemcpyAsync(ws.u[0], psi, D * esize(dtype), cudaMemcpyDeviceToDevice, st));
    RP_CUDA(cudaMemsetAsync(ws.y, 0, D * esize(dtype), st));
    RP_CUDA(cudaMemsetAsync(ws.err, 0, sizeof(unsigned), st));
    k_kry_init<<<1, 32, 0, st>>>(ws.dev, beta0);
    RP_CUDA(cudaGetLastError());

    // device copy of the pointer table for the fused projections of the apply
    void **d_tab = ws.tab;

    const bool fused = !plan.cfg.direct && fused_projections();
    const int agrid = fused ? apply_grid(plan) : reduce_grid();
    const int rgrid = reduce_grid();
    KryDev *s = ws.dev;
    int cycle = 0;
    KryHeader hdr{};
    while (true) {
        cycle++;
        grow_hfull(ws, cycle * krydim, st);
        k_kry_begin<<<1, 256, 0, st>>>(s, krydim, cycle > 1);
        VecTable tab{};
        for (int i = 0; i <= krydim; i++) tab.p[i] = ws.u[i];
        RP_CUDA(cudaMemcpyAsync(d_tab, tab.p, (krydim + 1) * sizeof(void *),
                                cudaMemcpyHostToDevice, st));
        for (int j = 0; j < krydim; j++) {
            void *w = ws.u[j + 1];
            ApplyLaunch L;
            L.in = ws.u[j];
            L.out = w;
            L.alpha_dev = &s->sigma[j];
            L.active = &s->active;
            L.err = ws.err;
            if (fused) {
                L.dot_vecs = (const void *const *)d_tab;
                L.ndot = j + 1;
                L.partials = ws.partials;
                apply_launch(plan, L, st);
            } else {
                apply_launch(plan, L, st);
                multi_dot_partials(dtype, D, tab, j + 1, w, ws.partials, &s->active, nullptr, st);
            }
            k_kry_proj<<<1, 256, 0, st>>>(s, ws.partials, agrid, j, 1);
            multi_axpy(dtype, D, tab, j + 1, nullptr, s->coef, w, ws.norm_partials, &s->active,
                       nullptr, st);
            k_kry_norm<<<1, 32, 0, st>>>(s, ws.norm_partials, rgrid, j, krydim, 1);
            for (int pass = 2; pass <= 3; pass++) {
                multi_dot_partials(dtype, D, tab, j + 1, w, ws.partials, &s->active, &s->again, st);
                k_kry_proj<<<1, 256, 0, st>>>(s, ws.partials, rgrid, j, pass);
                multi_axpy(dtype, D, tab, j + 1, nullptr, s->coef, w, ws.norm_partials,
                           &s->active, &s->again, st);
                k_kry_norm<<<1, 32, 0, st>>>(s, ws.norm_partials, rgrid, j, krydim, pass);
            }
        }
        const int n = cycle * krydim;
        const size_t smem = (size_t)(2 * n + 64) * sizeof(double);
        k_kry_expm<<<1, 512, smem, st>>>(s, (cd *)ws.hfull, ws.hcap, (cd *)ws.escratch, krydim,
                                         cycle, -t_imag, -t_real);
        RP_CUDA(cudaGetLastError());
        multi_axpy(dtype, D, tab, krydim, &s->m_eff, s->ycoef, ws.y, nullptr, nullptr, nullptr, st);
        unsigned herr = 0;
        RP_CUDA(cudaMemcpyAsync(&hdr, s, sizeof(hdr), cudaMemcpyDeviceToHost, st));
        RP_CUDA(cudaMemcpyAsync(&herr, ws.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        RP_CUDA(cudaStreamSynchronize(st));
        RP_REQUIRE(herr == 0, -5, "a device-side wait timed out in the H.psi kernel");
        S.restarts = cycle;
        S.applies += hdr.m_eff;
        S.last_err = hdr.nrm;
        if ((max_iters && cycle >= max_iters) || hdr.brokedown || hdr.nrm < tol) {
            S.breakdown = hdr.brokedown;
            break;
        }
        std::swap(ws.u[0], ws.u[krydim]);
    }
    S.passes = hdr.passes;
    S.prods = hdr.prods + 1;   // + the norm of the initial vector
    RP_CUDA(cudaMemcpyAsync(psi, ws.y, D * esize(dtype), cudaMemcpyDeviceToDevice, st));
    RP_CUDA(cudaStreamSynchronize(st));
    if (stats) *stats = S;
}

// ---------------------------------------------------------------------------
// Time-stepped primitives
// ---------------------------------------------------------------------------
void krylov_arnoldi(const ApplyPlan &plan, KryWorkspace &ws, const void *psi, int m,
                    ArnoldiResult &R, cudaStream_t st) {
    RP_REQUIRE(m >= 2 && m <= MAX_KRYLOV, -2, "m must be in [2, 64]");
    workspace_ensure(ws, plan.len, plan.dtype, m);
    const uint64_t D = ws.D;
    const int dtype = plan.dtype;
    R = ArnoldiResult{};
    R.m = m;
    R.beta0 = vec_norm_sync(dtype, D, psi, &ws, st);
    R.H.assign((size_t)2 * m * m, 0.0);
    R.sigma.assign(m + 1, 0.0);
    if (R.beta0 == 0.0) return;
    RP_CUDA(cudaMemcpyAsync(ws.u[0], psi, D * esize(dtype), cudaMemcpyDeviceToDevice, st));
    RP_CUDA(cudaMemsetAsync(ws.err, 0, sizeof(unsigned), st));
    k_kry_init<<<1, 32, 0, st>>>(ws.dev, R.beta0);
    k_kry_begin<<<1, 256, 0, st>>>(ws.dev, m, 0);
    RP_CUDA(cudaGetLastError());
    void **d_tab = ws.tab;
    VecTable tab{};
    for (int i = 0; i <= m; i++) tab.p[i] = ws.u[i];
    RP_CUDA(cudaMemcpyAsync(d_tab, tab.p, (m + 1) * sizeof(void *), cudaMemcpyHostToDevice, st));
    const bool fused = !plan.cfg.direct && fused_projections();
    const int agrid = fused ? apply_grid(plan) : reduce_grid();
    const int rgrid = reduce_grid();
    KryDev *s = ws.dev;
    for (int j = 0; j < m; j++) {
        void *w = ws.u[j + 1];
        ApplyLaunch L;
        L.in = ws.u[j];
        L.out = w;
        L.alpha_dev = &s->sigma[j];
        L.active = &s->active;
        L.err = ws.err;
        if (fused) {
            L.dot_vecs = (const void *const *)d_tab;
            L.ndot = j + 1;
            L.partials = ws.partials;
            apply_launch(plan, L, st);
        } else {
            apply_launch(plan, L, st);
            multi_dot_partials(dtype, D, tab, j + 1, w, ws.partials, &s->active, nullptr, st);
        }
        k_kry_proj<<<1, 256, 0, st>>>(s, ws.partials, agrid, j, 1);
        multi_axpy(dtype, D, tab, j + 1, nullptr, s->coef, w, ws.norm_partials, &s->active,
                   nullptr, st);
        k_kry_norm<<<1, 32, 0, st>>>(s, ws.norm_partials, rgrid, j, m, 1);
        for (int pass = 2; pass <= 3; pass++) {
            multi_dot_partials(dtype, D, tab, j + 1, w, ws.partials, &s->active, &s->again, st);
            k_kry_proj<<<1, 256, 0, st>>>(s, ws.partials, rgrid, j, pass);
            multi_axpy(dtype, D, tab, j + 1, nullptr, s->coef, w, ws.norm_partials, &s->active,
                       &s->again, st);
            k_kry_norm<<<1, 32, 0, st>>>(s, ws.norm_partials, rgrid, j, m, pass);
        }
    }
    RP_CUDA(cudaGetLastError());
    KryHeader hdr{};
    unsigned herr = 0;
    RP_CUDA(cudaMemcpyAsync(&hdr, s, sizeof(hdr), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaMemcpyAsync(R.H.data(), s->H, R.H.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaMemcpyAsync(R.sigma.data(), s->sigma, (m + 1) * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaMemcpyAsync(&herr, ws.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
    RP_REQUIRE(herr == 0, -5, "a device-side wait timed out in the H.psi kernel");
    R.m_eff = hdr.m_eff;
    R.breakdown = hdr.brokedown;
    R.passes = hdr.passes;
    R.beta = hdr.beta;
}

void krylov_combine(KryWorkspace &ws, const ArnoldiResult &R, const double *coef, void *out,
                    cudaStream_t st) {
    RP_REQUIRE(R.m_eff >= 1 && (int)ws.u.size() >= R.m_eff, -2, "no Arnoldi basis to combine");
    std::vector<double> c((size_t)2 * R.m_eff);
    for (int i = 0; i < R.m_eff; i++) {
        c[2 * i] = coef[2 * i] * R.sigma[i];
        c[2 * i + 1] = coef[2 * i + 1] * R.sigma[i];
    }
    RP_CUDA(cudaMemcpyAsync(ws.dev->ycoef, c.data(), c.size() * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    RP_CUDA(cudaMemsetAsync(out, 0, ws.D * esize(ws.dtype), st));
    VecTable tab{};
    for (int i = 0; i < R.m_eff; i++) tab.p[i] = ws.u[i];
    multi_axpy(ws.dtype, ws.D, tab, R.m_eff, nullptr, ws.dev->ycoef, out, nullptr, nullptr,
               nullptr, st);
    RP_CUDA(cudaStreamSynchronize(st));
}

__global__ void __launch_bounds__(256) k_expm_cands(int m, const cd *H, const double *fr,
                                                    const double *fi, cd *scratch, cd *col0) {
    extern __shared__ double smem[];
    const int c = blockIdx.x;
    cd *A = scratch + (size_t)c * 10 * m * m, *E = A + (size_t)m * m, *ws = E + (size_t)m * m;
    const cd f{fr[c], fi[c]};
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) A[e] = cmul(f, H[e]);
    __syncthreads();
    expm_block(m, A, E, ws, smem);
    for (int i = threadIdx.x; i < m; i += blockDim.x) col0[(size_t)c * m + i] = E[i];
}

void expm_candidates(int m, const double *H, int ncand, const double *fr, const double *fi,
                     double *col0, cudaStream_t st) {
    RP_REQUIRE(m >= 1 && m <= 1024 && ncand >= 1 && ncand <= 64, -2, "bad expm batch size");
    const size_t hb = (size_t)m * m * sizeof(cd);
    const size_t sb = (size_t)ncand * 10 * m * m * sizeof(cd);
    const size_t need = hb + sb + 2 * ncand * sizeof(double) + (size_t)ncand * m * sizeof(cd);
    // one buffer kept between calls (a step controller calls this every step)
    char *buf = static_cast<char *>(scratch_get(SCR_EXPM, need, st));
    cd *dH = (cd *)buf;
    cd *scr = (cd *)(buf + hb);
    double *dfr = (double *)(buf + hb + sb), *dfi = dfr + ncand;
    cd *dcol = (cd *)(dfi + ncand);
    RP_CUDA(cudaMemcpyAsync(dH, H, hb, cudaMemcpyHostToDevice, st));
    RP_CUDA(cudaMemcpyAsync(dfr, fr, ncand * sizeof(double), cudaMemcpyHostToDevice, st));
    RP_CUDA(cudaMemcpyAsync(dfi, fi, ncand * sizeof(double), cudaMemcpyHostToDevice, st));
    k_expm_cands<<<ncand, 256, (size_t)(2 * m + 64) * sizeof(double), st>>>(m, dH, dfr, dfi, scr, dcol);
    RP_CUDA(cudaGetLastError());
    RP_CUDA(cudaMemcpyAsync(col0, dcol, (size_t)ncand * m * sizeof(cd), cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
}

}  // namespace rp
