#pragma once
// Single-CTA FP64 matrix exponential (Higham 2005, Pade 3..13 with scaling
// and squaring), included into the translation unit that launches it.
// Matrices live in global scratch (L2-resident at Krylov
// sizes); every step is a block-wide loop with __syncthreads between steps.
#include "rp_expm.cuh"

namespace rp {

// Pade numerator coefficients b_0..b_m of Higham (2005), Table 2.2.
static __constant__ double c_b13[14] = {
    64764752532480000.0, 32382376266240000.0, 7771770303897600.0, 1187353796428800.0,
    129060195264000.0,   10559470521600.0,    670442572800.0,     33522128640.0,
    1323241920.0,        40840800.0,          960960.0,           16380.0,
    182.0,               1.0};
static __constant__ double c_b9[10] = {17643225600.0, 8821612800.0, 2075673600.0, 302702400.0,
                                30270240.0,    2162160.0,    110880.0,     3960.0,
                                90.0,          1.0};
static __constant__ double c_b7[8] = {17297280.0, 8648640.0, 1995840.0, 277200.0,
                               25200.0,    1512.0,    56.0,      1.0};
static __constant__ double c_b5[6] = {30240.0, 15120.0, 3360.0, 420.0, 30.0, 1.0};
static __constant__ double c_b3[4] = {120.0, 60.0, 12.0, 1.0};

// C = A * B (n x n), block-wide.
__device__ static void mm(int n, const cd *A, const cd *B, cd *C) {
    const int nn = n * n;
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
        const int i = e % n, j = e / n;
        double sr = 0.0, si = 0.0;
        for (int k = 0; k < n; k++) {
            const cd a = A[i + k * n], b = B[k + j * n];
            sr = fma(a.x, b.x, fma(-a.y, b.y, sr));
            si = fma(a.x, b.y, fma(a.y, b.x, si));
        }
        C[e] = cd{sr, si};
    }
    __syncthreads();
}

// Solve Q X = P in place (X -> P), Gaussian elimination with partial pivoting.
__device__ static void solve(int n, cd *Q, cd *P, double *smem) {
    double *fac = smem;              // 2n doubles: elimination factors
    __shared__ int s_piv;
    __shared__ double s_best[32];
    __shared__ int s_idx[32];
    for (int k = 0; k < n; k++) {
        // pivot search over rows k..n-1 of column k
        double best = -1.0;
        int bi = k;
        for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
            const cd q = Q[i + k * n];
            const double v = hypot(q.x, q.y);
            if (v > best) { best = v; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if ((threadIdx.x & 31) == 0) { s_best[threadIdx.x >> 5] = best; s_idx[threadIdx.x >> 5] = bi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = -1.0;
            int p = k;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++)
                if (s_best[w] > b || (s_best[w] == b && s_idx[w] < p)) { b = s_best[w]; p = s_idx[w]; }
            s_piv = p;
        }
        __syncthreads();
        const int p = s_piv;
        if (p != k) {
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                cd t = Q[k + j * n]; Q[k + j * n] = Q[p + j * n]; Q[p + j * n] = t;
                t = P[k + j * n]; P[k + j * n] = P[p + j * n]; P[p + j * n] = t;
            }
        }
        __syncthreads();
        const cd d = Q[k + k * n];
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
            const cd f = cdiv(Q[i + k * n], d);
            fac[2 * i] = f.x;
            fac[2 * i + 1] = f.y;
        }
        __syncthreads();
        const int rows = n - k - 1;
        for (int e = threadIdx.x; e < rows * 2 * n; e += blockDim.x) {
            const int i = k + 1 + e % rows;
            const int jj = e / rows;   // 0..2n-1: columns of Q then of P
            const cd f{fac[2 * i], fac[2 * i + 1]};
            if (jj < n) {
                if (jj >= k) {
                    const cd a = Q[k + jj * n], t = cmul(f, a);
                    Q[i + jj * n].x -= t.x;
                    Q[i + jj * n].y -= t.y;
                }
            } else {
                const int j = jj - n;
                const cd a = P[k + j * n], t = cmul(f, a);
                P[i + j * n].x -= t.x;
                P[i + j * n].y -= t.y;
            }
        }
        __syncthreads();
    }
    // back substitution, one column of P per thread group
    for (int i = n - 1; i >= 0; i--) {
        const cd d = Q[i + i * n];
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            double sr = P[i + j * n].x, si = P[i + j * n].y;
            for (int k = i + 1; k < n; k++) {
                const cd q = Q[i + k * n], x = P[k + j * n];
                sr -= q.x * x.x - q.y * x.y;
                si -= q.x * x.y + q.y * x.x;
            }
            P[i + j * n] = cdiv(cd{sr, si}, d);
        }
        __syncthreads();
    }
}

__device__ inline void expm_block(int n, const cd *A_in, cd *E, cd *scratch, double *smem) {
    const int nn = n * n;
    cd *A = scratch, *A2 = A + nn, *A4 = A2 + nn, *A6 = A4 + nn;
    cd *U = A6 + nn, *V = U + nn, *T = V + nn, *Pm = T + nn;
    __shared__ double s_norm;
    __shared__ double s_colmax[32];
    // 1-norm (max column sum of |a_ij|)
    double best = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < n; i++) s += hypot(A_in[i + j * n].x, A_in[i + j * n].y);
        best = fmax(best, s);
    }
    for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) s_colmax[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) b = fmax(b, s_colmax[w]);
        s_norm = b;
    }
    __syncthreads();
    const double a1 = s_norm;
    int deg, s = 0;
    if (a1 <= 1.495585217958292e-2) deg = 3;
    else if (a1 <= 2.539398330063230e-1) deg = 5;
    else if (a1 <= 9.504178996162932e-1) deg = 7;
    else if (a1 <= 2.097847961257068e0) deg = 9;
    else {
        deg = 13;
        const double r = a1 / 5.371920351148152e0;
        if (r > 1.0) s = (int)ceil(log2(r));
    }
    const double sc = ldexp(1.0, -s);
    for (int e = threadIdx.x; e < nn; e += blockDim.x) A[e] = cd{A_in[e].x * sc, A_in[e].y * sc};
    __syncthreads();
    mm(n, A, A, A2);
    if (deg == 13) {
        mm(n, A2, A2, A4);
        mm(n, A4, A2, A6);
        for (int e = threadIdx.x; e < nn; e += blockDim.x) {
            T[e] = cd{c_b13[13] * A6[e].x + c_b13[11] * A4[e].x + c_b13[9] * A2[e].x,
                      c_b13[13] * A6[e].y + c_b13[11] * A4[e].y + c_b13[9] * A2[e].y};
        }
        __syncthreads();
        mm(n, A6, T, Pm);
        for (int e = threadIdx.x; e < nn; e += blockDim.x) {
            const int i = e % n, j = e / n;
            cd p = Pm[e];
            p.x += c_b13[7] * A6[e].x + c_b13[5] * A4[e].x + c_b13[3] * A2[e].x + (i == j ? c_b13[1] : 0.0);
            p.y += c_b13[7] * A6[e].y + c_b13[5] * A4[e].y + c_b13[3] * A2[e].y;
            Pm[e] = p;
            T[e] = cd{c_b13[12] * A6[e].x + c_b13[10] * A4[e].x + c_b13[8] * A2[e].x,
                      c_b13[12] * A6[e].y + c_b13[10] * A4[e].y + c_b13[8] * A2[e].y};
        }
        __syncthreads();
        mm(n, A, Pm, U);
        mm(n, A6, T, V);
        for (int e = threadIdx.x; e < nn; e += blockDim.x) {
            const int i = e % n, j = e / n;
            cd v = V[e];
            v.x += c_b13[6] * A6[e].x + c_b13[4] * A4[e].x + c_b13[2] * A2[e].x + (i == j ? c_b13[0] : 0.0);
            v.y += c_b13[6] * A6[e].y + c_b13[4] * A4[e].y + c_b13[2] * A2[e].y;
            V[e] = v;
        }
        __syncthreads();
    } else {
        const double *b = deg == 3 ? c_b3 : deg == 5 ? c_b5 : deg == 7 ? c_b7 : c_b9;
        // Pm = A^(2k), accumulated into V (even part) and T (odd part / A)
        for (int e = threadIdx.x; e < nn; e += blockDim.x) {
            const int i = e % n, j = e / n;
            const double id = i == j ? 1.0 : 0.0;
            Pm[e] = cd{id, 0.0};
            V[e] = cd{b[0] * id, 0.0};
            T[e] = cd{b[1] * id, 0.0};
        }
        __syncthreads();
        for (int k = 1; 2 * k <= deg; k++) {
            mm(n, Pm, A2, A4);   // A4 as the next power
            for (int e = threadIdx.x; e < nn; e += blockDim.x) {
                const cd p = A4[e];
                Pm[e] = p;
                V[e].x += b[2 * k] * p.x;
                V[e].y += b[2 * k] * p.y;
                T[e].x += b[2 * k + 1] * p.x;
                T[e].y += b[2 * k + 1] * p.y;
            }
            __syncthreads();
        }
        mm(n, A, T, U);
    }
    // (V - U) X = (V + U)
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
        const cd u = U[e], v = V[e];
        T[e] = cd{v.x - u.x, v.y - u.y};
        Pm[e] = cd{v.x + u.x, v.y + u.y};
    }
    __syncthreads();
    solve(n, T, Pm, smem);
    for (int k = 0; k < s; k++) {
        mm(n, Pm, Pm, T);
        for (int e = threadIdx.x; e < nn; e += blockDim.x) Pm[e] = T[e];
        __syncthreads();
    }
    for (int e = threadIdx.x; e < nn; e += blockDim.x) E[e] = Pm[e];
    __syncthreads();
}

}  // namespace rp
