/*
 * rp_oracle.c -- CPU restatement of the REAPERS hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product in
 * reapers_b200/csrc.  Only tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg of bench.py load it; the product never links or calls it.
 *
 * What is restated (reference file:line, paths inside cl91/REAPERS):
 *   - Pauli-string encoding, 2 bits per site: bit 2i = X_i, bit 2i+1 = Z_i
 *     (inc/ops.h:138-143); sigma_y is stored as the real sx.sz product with
 *     the factor i folded into the coefficient (inc/ops.h:285-288).
 *   - SpinOp product with the carry-over minus sign (inc/ops.h:151-161,319-327).
 *   - SpinOp::apply: res = n ^ xmask, sign (-1)^popcount(zmask & (n ^ xmask))
 *     (inc/ops.h:421-440).
 *   - CPUImpl::apply_ops: res[i] += sum_k coeff_k * sign * vec[n], terms in list
 *     order (inc/cpuimpl.h:739-754).  The reference switches to a dense
 *     mat-vec when #terms >= 2^len (inc/cpuimpl.h:742-745); the sum is the same
 *     up to rounding, and the oracle always uses the sparse loop.
 *   - Krylov::orthogonalize (iterated MGS, eta = 1/sqrt 2, <= 3 passes,
 *     old_norm seeded with eta/2) (inc/algo.h:77-107).
 *   - Krylov::arnoldi (inc/algo.h:145-173).
 *   - Krylov::evolve, the Eiermann-Ernst restart with the growing block
 *     Hessenberg matrix (inc/algo.h:267-365).
 *   - Majorana operators in non-block Jordan-Wigner form
 *     (inc/fermions.h:276-296) and the SYK scale (inc/syk.h:104-119).
 *
 * Third-party arithmetic on the path: the reference takes the exponential of
 * the small Hessenberg matrix with Eigen's MatrixFunctions exp() (algo.h:332),
 * an unpinned dependency that is not vendored.  It is restated here from the
 * published method it implements: N. J. Higham, "The scaling and squaring
 * method for the matrix exponential revisited", SIAM J. Matrix Anal. Appl.
 * 26(4), 2005 -- Pade degrees 3/5/7/9/13 chosen by the 1-norm thresholds
 * theta_m of that paper's Table 2.3, with scaling and squaring for degree 13.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ---------------------------------------------------------------------------
 * Pauli strings
 * ------------------------------------------------------------------------- */

/* Split the interleaved representation into the X mask and the Z mask. */
void or_split_bits(uint64_t bits, uint32_t *x, uint32_t *z)
{
    uint32_t xm = 0, zm = 0;
    for (int i = 0; i < 32; i++) {
        if ((bits >> (2 * i)) & 1) xm |= 1u << i;
        if ((bits >> (2 * i + 1)) & 1) zm |= 1u << i;
    }
    *x = xm;
    *z = zm;
}

/* The four products of sigma matrices that carry a minus sign:
 * sz.sx, sz.sy, sy.sx, sy.sy  (inc/ops.h:151-161).  Codes: id=0, x=1, z=2, y=3. */
static int prod_has_minus(unsigned s0, unsigned s1)
{
    unsigned k = (s0 << 2) | s1;
    return k == 0x9 || k == 0xB || k == 0xD || k == 0xF;
}

/* (a_bits, a) * (b_bits, b): coefficient product with the carry-over sign,
 * bits combined by XOR (inc/ops.h:319-327). */
void or_spin_mul(uint64_t a_bits, const double *a, uint64_t b_bits, const double *b,
                 uint64_t *out_bits, double *out)
{
    int minus = 0;
    for (int i = 0; i < 32; i++) {
        unsigned sa = (unsigned)((a_bits >> (2 * i)) & 3);
        unsigned sb = (unsigned)((b_bits >> (2 * i)) & 3);
        if (sa && prod_has_minus(sa, sb)) minus = !minus;
    }
    cplx ca = a[0] + I * a[1];
    cplx cb = b[0] + I * b[1];
    cplx c = (minus ? -ca : ca) * cb;
    *out_bits = a_bits ^ b_bits;
    out[0] = creal(c);
    out[1] = cimag(c);
}

/* Majorana b_n of N fields in non-block form (inc/fermions.h:276-296):
 *   b_n = {sy or sz}((n-1)/2) . prod_{(n+1)/2 <= i < N/2} sx(i)
 * built by right-multiplying the identity with the sx factors first and the
 * sy/sz factor last, then divided by sqrt(2) for the standard normalisation. */
void or_majorana(int N, int n, int standard_gamma, uint64_t *bits, double *coeff)
{
    uint64_t b = 0;
    double c[2] = {1.0, 0.0};
    for (int i = (n + 1) / 2; i < N / 2; i++) {
        double one[2] = {1.0, 0.0};
        or_spin_mul(b, c, (uint64_t)1 << (2 * i), one, &b, c);
    }
    if (n != 0) {
        int site = (n - 1) / 2;
        if (n & 1) {
            double ii[2] = {0.0, 1.0};   /* sigma_y = i * (sx.sz) */
            or_spin_mul(b, c, (uint64_t)3 << (2 * site), ii, &b, c);
        } else {
            double one[2] = {1.0, 0.0};
            or_spin_mul(b, c, (uint64_t)2 << (2 * site), one, &b, c);
        }
    }
    if (standard_gamma) {
        /* SpinOp::operator/= multiplies by 1/s (inc/ops.h:272-275) */
        cplx s = 1.0 / (cplx)sqrt(2.0);
        cplx cc = (c[0] + I * c[1]) * s;
        c[0] = creal(cc);
        c[1] = cimag(cc);
    }
    *bits = b;
    coeff[0] = c[0];
    coeff[1] = c[1];
}

/* SYK coupling scale (inc/syk.h:104-119): sqrt(6/N^3) J for standard gamma,
 * divided by sqrt(p) with p = 24 sp / ((N-1)(N-2)(N-3)) when sparse. */
double or_syk_scale(int N, double sp, double J)
{
    double scale = sqrt(6.0 / ((double)N * N * N)) * J;
    if (sp != 0.0) {
        double p = sp * 24 / (double)((N - 1) * (N - 2) * (N - 3));
        scale /= sqrt(p);
    }
    return scale;
}

/* Quartic SYK terms: term q = J_q * b_i b_j b_k b_l for quartets (i,j,k,l)
 * with i>j>k>l, products taken left to right as gen_ham does
 * (inc/syk.h:254-256).  J_q already includes the scale.  Writes T entries. */
void or_syk_terms(int N, int T, const int *quartets, const double *J,
                  uint64_t *bits, double *coeff)
{
    for (int q = 0; q < T; q++) {
        uint64_t b;
        double c[2] = {J[q], 0.0};
        b = 0;
        for (int f = 0; f < 4; f++) {
            uint64_t mb;
            double mc[2];
            or_majorana(N, quartets[4 * q + f], 1, &mb, mc);
            or_spin_mul(b, c, mb, mc, &b, c);
        }
        bits[q] = b;
        coeff[2 * q] = c[0];
        coeff[2 * q + 1] = c[1];
    }
}

/* ---------------------------------------------------------------------------
 * H.psi
 * ------------------------------------------------------------------------- */

/* out[i] (+)= sum_k c_k (-1)^popc(z_k & (i ^ x_k)) in[i ^ x_k], in list order
 * (inc/cpuimpl.h:747-753 with SpinOp::apply, inc/ops.h:421-440). */
void or_apply(int len, int64_t T, const uint64_t *bits, const double *coeff,
              const double *in, double *out, int accumulate)
{
    uint64_t D = (uint64_t)1 << len;
    uint32_t *xs = malloc(sizeof(uint32_t) * (T ? T : 1));
    uint32_t *zs = malloc(sizeof(uint32_t) * (T ? T : 1));
    for (int64_t k = 0; k < T; k++) or_split_bits(bits[k], &xs[k], &zs[k]);
    const cplx *vin = (const cplx *)in;
    cplx *vout = (cplx *)out;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)D; i++) {
        cplx acc = accumulate ? vout[i] : 0.0;
        for (int64_t k = 0; k < T; k++) {
            uint32_t n = (uint32_t)i ^ xs[k];
            int minus = __builtin_popcount(zs[k] & n) & 1;
            cplx c = coeff[2 * k] + I * coeff[2 * k + 1];
            acc += (minus ? -c : c) * vin[n];
        }
        vout[i] = acc;
    }
    free(xs);
    free(zs);
}

/* ---------------------------------------------------------------------------
 * Dense complex helpers (column-major n x n)
 * ------------------------------------------------------------------------- */

static void mat_mul(int n, const cplx *A, const cplx *B, cplx *C)
{
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < n; i++) C[i + j * n] = 0;
        for (int k = 0; k < n; k++) {
            cplx b = B[k + j * n];
            if (b == 0) continue;
            for (int i = 0; i < n; i++) C[i + j * n] += A[i + k * n] * b;
        }
    }
}

static double norm1(int n, const cplx *A)
{
    double best = 0;
    for (int j = 0; j < n; j++) {
        double s = 0;
        for (int i = 0; i < n; i++) s += cabs(A[i + j * n]);
        if (s > best) best = s;
    }
    return best;
}

/* Solve Q X = P in place (P overwritten by X), Gaussian elimination with
 * partial pivoting.  Returns 0 on success. */
static int solve(int n, cplx *Q, cplx *P)
{
    int *piv = malloc(sizeof(int) * n);
    for (int k = 0; k < n; k++) {
        int p = k;
        double best = cabs(Q[k + k * n]);
        for (int i = k + 1; i < n; i++) {
            double v = cabs(Q[i + k * n]);
            if (v > best) { best = v; p = i; }
        }
        if (best == 0) { free(piv); return -1; }
        piv[k] = p;
        if (p != k) {
            for (int j = 0; j < n; j++) {
                cplx t = Q[k + j * n]; Q[k + j * n] = Q[p + j * n]; Q[p + j * n] = t;
                t = P[k + j * n]; P[k + j * n] = P[p + j * n]; P[p + j * n] = t;
            }
        }
        cplx d = Q[k + k * n];
        for (int i = k + 1; i < n; i++) {
            cplx f = Q[i + k * n] / d;
            if (f == 0) continue;
            for (int j = k; j < n; j++) Q[i + j * n] -= f * Q[k + j * n];
            for (int j = 0; j < n; j++) P[i + j * n] -= f * P[k + j * n];
        }
    }
    for (int j = 0; j < n; j++) {
        for (int i = n - 1; i >= 0; i--) {
            cplx s = P[i + j * n];
            for (int k = i + 1; k < n; k++) s -= Q[i + k * n] * P[k + j * n];
            P[i + j * n] = s / Q[i + i * n];
        }
    }
    free(piv);
    return 0;
}

/* Pade coefficients b_0..b_13 of Higham (2005), eq. (2.11) / Table 2.2. */
static const double pade13[14] = {
    64764752532480000.0, 32382376266240000.0, 7771770303897600.0,
    1187353796428800.0, 129060195264000.0, 10559470521600.0, 670442572800.0,
    33522128640.0, 1323241920.0, 40840800.0, 960960.0, 16380.0, 182.0, 1.0};
static const double pade9[10] = {17643225600.0, 8821612800.0, 2075673600.0,
    302702400.0, 30270240.0, 2162160.0, 110880.0, 3960.0, 90.0, 1.0};
static const double pade7[8] = {17297280.0, 8648640.0, 1995840.0, 277200.0,
    25200.0, 1512.0, 56.0, 1.0};
static const double pade5[6] = {30240.0, 15120.0, 3360.0, 420.0, 30.0, 1.0};
static const double pade3[4] = {120.0, 60.0, 12.0, 1.0};

/* E = exp(A), n x n complex column-major, by Higham's scaling and squaring.
 * Returns 0 on success. */
int or_expm(int n, const double *Ain, double *Eout)
{
    size_t nn = (size_t)n * n;
    cplx *A = malloc(sizeof(cplx) * nn);
    memcpy(A, Ain, sizeof(cplx) * nn);
    cplx *A2 = malloc(sizeof(cplx) * nn), *A4 = malloc(sizeof(cplx) * nn);
    cplx *A6 = malloc(sizeof(cplx) * nn), *U = malloc(sizeof(cplx) * nn);
    cplx *V = malloc(sizeof(cplx) * nn), *T = malloc(sizeof(cplx) * nn);
    cplx *P = malloc(sizeof(cplx) * nn), *Q = malloc(sizeof(cplx) * nn);
    double a1 = norm1(n, A);
    const double theta[5] = {1.495585217958292e-2, 2.539398330063230e-1,
                             9.504178996162932e-1, 2.097847961257068e0,
                             5.371920351148152e0};
    int s = 0;
    int deg;
    if (a1 <= theta[0]) deg = 3;
    else if (a1 <= theta[1]) deg = 5;
    else if (a1 <= theta[2]) deg = 7;
    else if (a1 <= theta[3]) deg = 9;
    else {
        deg = 13;
        double r = a1 / theta[4];
        if (r > 1) s = (int)ceil(log2(r));
        double sc = ldexp(1.0, -s);
        for (size_t i = 0; i < nn; i++) A[i] *= sc;
    }
    mat_mul(n, A, A, A2);
    memset(U, 0, sizeof(cplx) * nn);
    memset(V, 0, sizeof(cplx) * nn);
    if (deg == 13) {
        const double *b = pade13;
        mat_mul(n, A2, A2, A4);
        mat_mul(n, A4, A2, A6);
        /* U = A [A6 (b13 A6 + b11 A4 + b9 A2) + b7 A6 + b5 A4 + b3 A2 + b1 I] */
        for (size_t i = 0; i < nn; i++) T[i] = b[13] * A6[i] + b[11] * A4[i] + b[9] * A2[i];
        mat_mul(n, A6, T, P);
        for (size_t i = 0; i < nn; i++) P[i] += b[7] * A6[i] + b[5] * A4[i] + b[3] * A2[i];
        for (int i = 0; i < n; i++) P[i + i * n] += b[1];
        mat_mul(n, A, P, U);
        /* V = A6 (b12 A6 + b10 A4 + b8 A2) + b6 A6 + b4 A4 + b2 A2 + b0 I */
        for (size_t i = 0; i < nn; i++) T[i] = b[12] * A6[i] + b[10] * A4[i] + b[8] * A2[i];
        mat_mul(n, A6, T, V);
        for (size_t i = 0; i < nn; i++) V[i] += b[6] * A6[i] + b[4] * A4[i] + b[2] * A2[i];
        for (int i = 0; i < n; i++) V[i + i * n] += b[0];
    } else {
        const double *b = deg == 3 ? pade3 : deg == 5 ? pade5 : deg == 7 ? pade7 : pade9;
        /* powers A^0, A^2, A^4, ... accumulated into Uo (odd part) and V */
        cplx *Pk = malloc(sizeof(cplx) * nn);
        memset(Pk, 0, sizeof(cplx) * nn);
        for (int i = 0; i < n; i++) Pk[i + i * n] = 1.0;
        memset(T, 0, sizeof(cplx) * nn);
        for (int k = 0; 2 * k <= deg; k++) {
            for (size_t i = 0; i < nn; i++) {
                V[i] += b[2 * k] * Pk[i];
                T[i] += b[2 * k + 1] * Pk[i];
            }
            if (2 * k + 2 <= deg) {
                mat_mul(n, Pk, A2, P);
                memcpy(Pk, P, sizeof(cplx) * nn);
            }
        }
        mat_mul(n, A, T, U);
        free(Pk);
    }
    /* (V - U) E = (V + U) */
    for (size_t i = 0; i < nn; i++) {
        Q[i] = V[i] - U[i];
        P[i] = V[i] + U[i];
    }
    int rc = solve(n, Q, P);
    for (int k = 0; k < s; k++) {
        mat_mul(n, P, P, T);
        memcpy(P, T, sizeof(cplx) * nn);
    }
    memcpy(Eout, P, sizeof(cplx) * nn);
    free(A); free(A2); free(A4); free(A6); free(U); free(V); free(T); free(P); free(Q);
    return rc;
}

/* ---------------------------------------------------------------------------
 * Restarted Krylov exp(-(t_imag + i t_real) H) psi
 * ------------------------------------------------------------------------- */

static cplx vdot(uint64_t D, const cplx *a, const cplx *b)
{
    double re = 0, im = 0;
    #pragma omp parallel for reduction(+:re,im) schedule(static)
    for (int64_t i = 0; i < (int64_t)D; i++) {
        cplx r = conj(a[i]) * b[i];
        re += creal(r);
        im += cimag(r);
    }
    return re + I * im;
}

static void vaxpy(uint64_t D, cplx *y, cplx a, const cplx *x)
{
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)D; i++) y[i] += a * x[i];
}

static void vscale(uint64_t D, cplx *y, double a)
{
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)D; i++) y[i] *= a;
}

/* Krylov::orthogonalize (inc/algo.h:77-107).  V[0..j] orthonormal, V[j+1] is
 * the vector to orthogonalise.  Writes column j of H (ld = ldh) and *beta.
 * Returns 1 when the vector is linearly independent. */
static int orthogonalize(uint64_t D, cplx **V, cplx *H, int ldh, int j,
                         double *beta, int *passes, int *prods)
{
    const double eta = 1.0 / sqrt(2.0);
    cplx *h = calloc(j + 1, sizeof(cplx));
    double old_norm = 1.0, norm = eta / 2;
    int niter = 0;
    while (niter < 3 && norm != 0 && norm < eta * old_norm) {
        niter++;
        for (int i = 0; i <= j; i++) {
            cplx a = vdot(D, V[i], V[j + 1]);
            h[i] += a;
            vaxpy(D, V[j + 1], -a, V[i]);
        }
        old_norm = norm;
        norm = sqrt(creal(vdot(D, V[j + 1], V[j + 1])));
    }
    *beta = norm;
    for (int i = 0; i <= j; i++) H[i + j * ldh] = h[i];
    free(h);
    if (passes) *passes += niter;
    if (prods) *prods += niter * (j + 2);   /* j+1 projections and one norm per pass */
    return norm != 0 && norm >= eta * old_norm;
}

/* Statistics of one evolve call. */
typedef struct {
    int restarts;       /* Arnoldi cycles run */
    int applies;        /* H.psi products */
    int passes;         /* orthogonalisation passes */
    int prods;          /* inner products, norms included (vec_prod calls) */
    int breakdown;      /* 1 if an invariant subspace stopped the loop */
    double last_err;    /* ||Hexp0|| of the final cycle */
} or_evolve_stats;

/* psi <- exp(-(t_imag + i t_real) H) psi by Krylov::evolve (inc/algo.h:267-365).
 * psi is complex128 interleaved, length 2^len. */
int or_krylov_evolve(int len, int64_t T, const uint64_t *bits, const double *coeff,
                     double *psi_io, double t_real, double t_imag, int krydim,
                     double tol, int max_iters, or_evolve_stats *st)
{
    if (krydim < 2) return -1;
    uint64_t D = (uint64_t)1 << len;
    cplx *psi = (cplx *)psi_io;
    cplx **V = malloc(sizeof(cplx *) * (krydim + 1));
    for (int i = 0; i <= krydim; i++) V[i] = malloc(sizeof(cplx) * D);
    cplx *y = calloc(D, sizeof(cplx));
    memcpy(V[0], psi, sizeof(cplx) * D);
    double beta0 = sqrt(creal(vdot(D, V[0], V[0])));
    vscale(D, V[0], 1.0 / beta0);

    int cap = krydim * 8;
    cplx *Hfull = calloc((size_t)cap * cap, sizeof(cplx));
    int hdim = 0;
    double oldbeta = 0;
    int niters = 0;
    or_evolve_stats s = {0};
    s.prods = 1;   /* the norm of the initial vector */
    int rc = 0;
    cplx *H = malloc(sizeof(cplx) * krydim * krydim);
    while (1) {
        niters++;
        int m = krydim;
        double beta = 0;
        memset(H, 0, sizeof(cplx) * krydim * krydim);
        /* Krylov::arnoldi with k = 0 (inc/algo.h:145-173) */
        int brokedown = 0;
        for (int j = 0; j < m; j++) {
            or_apply(len, T, bits, coeff, (const double *)V[j], (double *)V[j + 1], 0);
            s.applies++;
            int ok = orthogonalize(D, V, H, krydim, j, &beta, &s.passes, &s.prods);
            if (!ok) {
                m = j + 1;
                brokedown = 1;
                break;
            }
            if (j != m - 1) H[(j + 1) + j * krydim] = beta;
            vscale(D, V[j + 1], 1.0 / beta);
        }
        /* grow Hfull: [OldHfull 0; 0..0 oldbeta H] (inc/algo.h:303-328) */
        int base = (niters - 1) * krydim;
        int ndim = base + m;
        if (ndim > cap) {
            int ncap = cap;
            while (ncap < ndim) ncap *= 2;
            cplx *nh = calloc((size_t)ncap * ncap, sizeof(cplx));
            for (int c = 0; c < hdim; c++)
                for (int r = 0; r < hdim; r++) nh[r + c * ncap] = Hfull[r + c * cap];
            free(Hfull);
            Hfull = nh;
            cap = ncap;
        }
        for (int c = 0; c < ndim; c++)
            for (int r = 0; r < ndim; r++)
                if (r >= base || c >= base) Hfull[r + c * cap] = 0;
        if (niters > 1) Hfull[base + (base - 1) * cap] = oldbeta;
        for (int c = 0; c < m; c++)
            for (int r = 0; r < m; r++) Hfull[(base + r) + (base + c) * cap] = H[r + c * krydim];
        hdim = ndim;
        /* Hexp = exp(-(t_imag + i t_real) Hfull) */
        cplx f = -t_imag - I * t_real;
        cplx *tH = malloc(sizeof(cplx) * hdim * hdim);
        cplx *E = malloc(sizeof(cplx) * hdim * hdim);
        for (int c = 0; c < hdim; c++)
            for (int r = 0; r < hdim; r++) tH[r + c * hdim] = f * Hfull[r + c * cap];
        or_expm(hdim, (const double *)tH, (double *)E);
        double nrm2 = 0;
        for (int i = 0; i < m; i++) {
            cplx e = E[base + i];   /* column 0, rows base..base+m-1 */
            vaxpy(D, y, beta0 * e, V[i]);
            nrm2 += creal(e) * creal(e) + cimag(e) * cimag(e);
        }
        free(tH);
        free(E);
        double nrm = sqrt(nrm2);
        s.last_err = nrm;
        s.restarts = niters;
        if ((max_iters && niters >= max_iters) || brokedown || nrm < tol) {
            s.breakdown = brokedown;
            break;
        }
        /* restart from v_m: swap_bufs(0, krydim) */
        cplx *tmp = V[0];
        V[0] = V[krydim];
        V[krydim] = tmp;
        oldbeta = beta;
    }
    memcpy(psi, y, sizeof(cplx) * D);
    for (int i = 0; i <= krydim; i++) free(V[i]);
    free(V);
    free(y);
    free(H);
    free(Hfull);
    if (st) *st = s;
    return rc;
}

/* Dense 2^len x 2^len matrix of the operator sum, column-major complex128.
 * Same entries as HostSumOps::get_matrix (inc/cpuimpl.h:372-390). */
void or_dense_matrix(int len, int64_t T, const uint64_t *bits, const double *coeff,
                     double *mat)
{
    uint64_t D = (uint64_t)1 << len;
    cplx *M = (cplx *)mat;
    memset(M, 0, sizeof(cplx) * D * D);
    for (int64_t k = 0; k < T; k++) {
        uint32_t x, z;
        or_split_bits(bits[k], &x, &z);
        cplx c = coeff[2 * k] + I * coeff[2 * k + 1];
        for (uint64_t i = 0; i < D; i++) {
            uint32_t n = (uint32_t)i ^ x;
            int minus = __builtin_popcount(z & n) & 1;
            M[i + (uint64_t)n * D] += minus ? -c : c;
        }
    }
}
