// FP64 exponential of a small dense complex matrix, computed by one CTA.
//
// Method: N. J. Higham, "The scaling and squaring method for the matrix
// exponential revisited", SIAM J. Matrix Anal. Appl. 26(4):1179-1193, 2005.
// The Pade degree m in {3,5,7,9,13} is the smallest whose 1-norm bound
// theta_m covers ||A||_1; above theta_13 the matrix is scaled by 2^-s and
// the result squared s times.  The reference computes this exponential with
// Eigen's MatrixFunctions exp() (inc/algo.h:331-332), which implements the
// same published method.
#pragma once

#include "rp_common.cuh"

namespace rp {

struct cd {
    double x, y;
};

__device__ __forceinline__ cd cmul(cd a, cd b) {
    return cd{fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x)};
}
__device__ __forceinline__ cd cdiv(cd a, cd b) {
    // Smith's algorithm
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return cd{(a.x + a.y * r) / d, (a.y - a.x * r) / d};
    } else {
        double r = b.x / b.y, d = b.x * r + b.y;
        return cd{(a.x * r + a.y) / d, (a.y * r - a.x) / d};
    }
}

// Scratch needed by expm_block for an n x n matrix (in cd elements).
__host__ __device__ inline size_t expm_scratch_elems(int n) { return (size_t)8 * n * n; }

// E = exp(A); A and E are n x n column-major with leading dimension n.
// Must be called by all threads of one CTA (blockDim.x a multiple of 32,
// at most 1024).  scratch holds expm_scratch_elems(n) elements; smem holds
// at least 2 * n + 64 doubles of dynamic shared memory.
__device__ inline void expm_block(int n, const cd *A, cd *E, cd *scratch, double *smem);

}  // namespace rp
