// Vector kernels (the BLAS-1 surface of the reference's Impl concept,
// inc/gpuimpl.h:853-1002) and the multi-vector kernels of block Gram-Schmidt.
#pragma once

#include "rp_common.cuh"

namespace rp {

constexpr int MAX_KRYLOV = 64;   // largest Krylov dimension (vectors u_0..u_m)

// Pointer table passed by value (kernel parameter space).
struct VecTable {
    const void *p[MAX_KRYLOV + 1];
};

// Grid used by the reduction kernels; partial buffers hold grid * n * 2 doubles.
int reduce_grid();

void vec_convert(int dtype_dst, void *dst, int dtype_src, const void *src, uint64_t n,
                 cudaStream_t st);
void vec_axpy(int dtype, uint64_t n, void *y, double ar, double ai, const void *x,
              cudaStream_t st);
void vec_add3(int dtype, uint64_t n, void *res, const void *a, const void *b, cudaStream_t st);
void vec_scale(int dtype, uint64_t n, void *v, double ar, double ai, cudaStream_t st);
void vec_random(int dtype, uint64_t n, void *v, uint64_t seed, cudaStream_t st);

// partials[cta][i][2] = per-CTA compensated partial of <u_i | w>, i < nvec
// (u_i = tab.p[i]).  Skipped when *gate == 0 or *gate2 == 0 (either may be null).
void multi_dot_partials(int dtype, uint64_t n, const VecTable &tab, int nvec, const void *w,
                        double *partials, const int *gate, const int *gate2, cudaStream_t st);

// w += sum_i coef[i] * u_i (coef complex double on the device), i < nvec or
// i < *nvec_dev when nvec_dev is given; partial ||w||^2 per CTA into
// norm_partials when non-null.  Skipped when a gate is 0.
void multi_axpy(int dtype, uint64_t n, const VecTable &tab, int nvec, const int *nvec_dev,
                const double *coef, void *w, double *norm_partials, const int *gate,
                const int *gate2, cudaStream_t st);

// Fixed-order compensated reduction of partials[grid][n][2] into out[n][2].
void reduce_partials(const double *partials, int grid, int n, double *out, cudaStream_t st);

// Device scratch kept between calls: the per-CTA partials of the one-off
// inner product and norm, the step-size candidates' expm buffer, the dense
// matrix-vector product's column-chunk partials and the dense exponential's
// scaled eigenvectors.  A slot
// grows on demand (the stream is synchronised before a smaller buffer is
// freed); scratch_release_all(), called by rp_shutdown, frees every slot, so
// a later rp_init allocates them afresh.
enum ScratchSlot { SCR_DOT = 0, SCR_NORM, SCR_EXPM, SCR_MATVEC, SCR_EXPM_DENSE, SCR_COUNT };
void *scratch_get(int slot, size_t bytes, cudaStream_t st);
void scratch_release_all();

}  // namespace rp
