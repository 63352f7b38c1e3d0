// Restarted Krylov exp(-(beta + i t) H) psi on the GPU.
#pragma once

#include <vector>

#include "rp_apply.cuh"
#include "rp_vec.cuh"

namespace rp {

// Device-resident control state of one evolve.  Vectors u_i are stored
// unnormalised; the Arnoldi basis is v_i = sigma[i] * u_i, so no separate
// normalisation pass is ever made.
struct KryDev {
    int active;      // the current Arnoldi cycle is still running
    int again;       // another orthogonalisation pass is due for this step
    int niter;       // passes made for the current step
    int m_eff;       // basis size of the cycle (krydim unless breakdown)
    int brokedown;   // invariant subspace found
    int passes;      // total orthogonalisation passes (statistics)
    int prods;       // inner products the reference's MGS would take (statistics)
    int pad;
    double norm, old_norm, beta, oldbeta, beta0, nrm;
    double sigma[MAX_KRYLOV + 1];
    double hacc[2 * (MAX_KRYLOV + 1)];    // column j of H accumulated over passes
    double coef[2 * (MAX_KRYLOV + 1)];    // update coefficients of the current pass
    double ycoef[2 * (MAX_KRYLOV + 1)];   // beta0 * Hexp0_i * sigma_i
    double H[2 * MAX_KRYLOV * MAX_KRYLOV];   // cycle Hessenberg matrix, column-major
};

struct EvolveStats {
    int restarts;
    int applies;
    int passes;
    int prods;
    int breakdown;
    double last_err;
};

// Workspace of one evolve: krydim+1 basis vectors, the answer, the device
// state and the reduction buffers.
struct KryWorkspace {
    int len = 0, dtype = 0, krydim = 0;
    uint64_t D = 0;
    std::vector<void *> u;
    void *y = nullptr;
    KryDev *dev = nullptr;
    double *partials = nullptr;
    double *norm_partials = nullptr;
    int hcap = 0;            // capacity (dimension) of Hfull
    void *hfull = nullptr;   // hcap x hcap complex double
    void *escratch = nullptr;
    unsigned *err = nullptr;
    void **tab = nullptr;    // device copy of the basis pointer table
};

// At least krydim + 1 basis vectors for states of 2^len elements of dtype:
// a workspace for the same state shape is kept and grown, never shrunk
// (rp_workspace_release frees it).
void workspace_ensure(KryWorkspace &ws, int len, int dtype, int krydim);
void workspace_release(KryWorkspace &ws);

// psi <- exp(-(t_imag + i t_real) H) psi, restarted Arnoldi with the
// Eiermann-Ernst update (inc/algo.h:267-365).  psi is a device vector of the
// plan's precision.
void krylov_evolve(const ApplyPlan &plan, KryWorkspace &ws, void *psi, double t_real,
                   double t_imag, int krydim, double tol, int max_iters, EvolveStats *stats,
                   cudaStream_t st);

// sqrt(<v|v>) (compensated FP64), synchronous.
double vec_norm_sync(int dtype, uint64_t n, const void *v, KryWorkspace *ws, cudaStream_t st);

// --- time-stepped Krylov primitives (used by the step controllers) -------
// One Arnoldi cycle of psi with m vectors, the reference's orthogonalisation
// (inc/algo.h:77-173): the basis stays in the workspace; H (m x m complex,
// column-major), the last norm beta = h_{m+1,m}, beta0 = ||psi|| and the
// basis scales come back to the host.
struct ArnoldiResult {
    int m = 0, m_eff = 0, breakdown = 0, passes = 0;
    double beta = 0, beta0 = 0;
    std::vector<double> H;       // 2 * m * m
    std::vector<double> sigma;   // m + 1
};
void krylov_arnoldi(const ApplyPlan &plan, KryWorkspace &ws, const void *psi, int m,
                    ArnoldiResult &R, cudaStream_t st);
// out = sum_{i < m_eff} coef_i v_i over the last basis (coef complex, host).
void krylov_combine(KryWorkspace &ws, const ArnoldiResult &R, const double *coef, void *out,
                    cudaStream_t st);
// col0[c] = first column of exp(f_c H) for ncand factors f_c = fr[c] + i fi[c]
// (FP64 Pade-13 on the GPU, one CTA per candidate).
void expm_candidates(int m, const double *H, int ncand, const double *fr, const double *fi,
                     double *col0, cudaStream_t st);

}  // namespace rp
