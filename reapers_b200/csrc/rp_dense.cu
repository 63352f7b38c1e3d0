// Exact diagonalisation on the device: the dense path of the reference's GPU
// backend (DevSumOps::get_matrix / get_eigensystem / _matexp,
// inc/gpuimpl.h:1180-1263; used by ExactDiagonalization, inc/algo.h:29-54).
//
// * The dense matrix of a Pauli sum is written column by column from the
//   term table: column m holds c_k (-1)^popc(z_k & m) in row m ^ x_k for
//   every term k (the SpinOp::apply rule, inc/ops.h:421-440), one thread per
//   column, so no two threads touch one element.
// * Its eigensystem comes from the library eigensolver (cuSOLVER heevd,
//   lower triangle, as the reference), eigenvalues ascending.
// * exp(c H) = V diag(e^{c lambda}) V^H: the columns of V scaled by a kernel,
//   then one library GEMM with V^H.
// * The dense matrix-vector product (mat_mul) is this file's own kernel: the
//   columns split into chunks over a 2-D grid, FP64 partial sums per chunk,
//   a second kernel adding the chunks in a fixed order.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <vector>

#include "rp_dense.cuh"
#include "rp_vec.cuh"

namespace rp {

static size_t esz(int dtype) { return dtype == 2 ? 16 : 8; }

template <typename Real>
__global__ void k_dense_build(Cplx<Real> *M, uint64_t dim, const DenseTerm *terms, int nterms) {
    const uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (m >= dim) return;
    Cplx<Real> *col = M + m * dim;
    for (int k = 0; k < nterms; k++) {
        const DenseTerm t = terms[k];
        const uint64_t row = m ^ t.x;
        const double s = (__popcll(t.z & m) & 1) ? -1.0 : 1.0;
        Cplx<Real> v = col[row];
        v.x = (Real)((double)v.x + s * t.cr);
        v.y = (Real)((double)v.y + s * t.ci);
        col[row] = v;
    }
}

// tmp[:, j] = V[:, j] * exp(c lambda_j)
template <typename Real>
__global__ void k_scale_cols(Cplx<Real> *tmp, const Cplx<Real> *V, const Real *lam, uint64_t dim,
                             double cr, double ci) {
    const uint64_t n = dim * dim;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = e / dim;
        const double l = (double)lam[j];
        const double mag = exp(cr * l);
        double sn, cs;
        sincos(ci * l, &sn, &cs);
        const double fr = mag * cs, fi = mag * sn;
        const Cplx<Real> v = V[e];
        tmp[e] = Cplx<Real>{(Real)(fr * v.x - fi * v.y), (Real)(fr * v.y + fi * v.x)};
    }
}

constexpr int MV_ROWS = 256;     // rows per block (threads)
constexpr int MV_CHUNKS = 32;    // column chunks (grid y)

template <typename Real>
__global__ void __launch_bounds__(MV_ROWS)
    k_matvec_part(const Cplx<Real> *M, uint64_t dim, const Cplx<Real> *v, double *part,
                  uint64_t cols_per_chunk) {
    const uint64_t i = blockIdx.x * (uint64_t)MV_ROWS + threadIdx.x;
    const uint64_t j0 = blockIdx.y * cols_per_chunk;
    const uint64_t j1 = j0 + cols_per_chunk < dim ? j0 + cols_per_chunk : dim;
    if (i >= dim) return;
    double ar = 0.0, ai = 0.0;
    for (uint64_t j = j0; j < j1; j++) {
        const Cplx<Real> a = M[i + j * dim], x = v[j];
        ar = fma((double)a.x, (double)x.x, fma(-(double)a.y, (double)x.y, ar));
        ai = fma((double)a.x, (double)x.y, fma((double)a.y, (double)x.x, ai));
    }
    part[(blockIdx.y * dim + i) * 2] = ar;
    part[(blockIdx.y * dim + i) * 2 + 1] = ai;
}

template <typename Real>
__global__ void k_matvec_sum(const double *part, uint64_t dim, int chunks, Cplx<Real> *res) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= dim) return;
    double ar = 0.0, ai = 0.0;
    for (int c = 0; c < chunks; c++) {
        ar += part[(c * dim + i) * 2];
        ai += part[(c * dim + i) * 2 + 1];
    }
    res[i] = Cplx<Real>{(Real)ar, (Real)ai};
}

void dense_matvec(int dtype, uint64_t dim, const void *M, const void *v, void *res,
                  cudaStream_t st) {
    if (!dim) return;
    const int chunks = (int)std::min<uint64_t>(MV_CHUNKS, (dim + 63) / 64);
    const uint64_t per = (dim + chunks - 1) / chunks;
    double *part = static_cast<double *>(
        scratch_get(SCR_MATVEC, (size_t)chunks * dim * 2 * sizeof(double), st));
    const dim3 grid((unsigned)((dim + MV_ROWS - 1) / MV_ROWS), (unsigned)chunks);
    const unsigned sb = (unsigned)((dim + 255) / 256);
    if (dtype == 2) {
        k_matvec_part<double><<<grid, MV_ROWS, 0, st>>>(static_cast<const Cplx<double> *>(M), dim,
                                                        static_cast<const Cplx<double> *>(v), part, per);
        k_matvec_sum<double><<<sb, 256, 0, st>>>(part, dim, chunks, static_cast<Cplx<double> *>(res));
    } else {
        k_matvec_part<float><<<grid, MV_ROWS, 0, st>>>(static_cast<const Cplx<float> *>(M), dim,
                                                       static_cast<const Cplx<float> *>(v), part, per);
        k_matvec_sum<float><<<sb, 256, 0, st>>>(part, dim, chunks, static_cast<Cplx<float> *>(res));
    }
    RP_CUDA(cudaGetLastError());
}

#define RP_SOLVER(call)                                                                     \
    do {                                                                                    \
        cusolverStatus_t s_ = (call);                                                       \
        if (s_ != CUSOLVER_STATUS_SUCCESS)                                                  \
            throw ::rp::Error{-3, std::string(#call) + " failed (" + std::to_string((int)s_) + ")"}; \
    } while (0)
#define RP_BLAS(call)                                                                       \
    do {                                                                                    \
        cublasStatus_t s_ = (call);                                                         \
        if (s_ != CUBLAS_STATUS_SUCCESS)                                                    \
            throw ::rp::Error{-3, std::string(#call) + " failed (" + std::to_string((int)s_) + ")"}; \
    } while (0)

static cusolverDnHandle_t g_solver = nullptr;
static cublasHandle_t g_blas = nullptr;

static void ensure_handles(cudaStream_t st) {
    if (!g_solver) RP_SOLVER(cusolverDnCreate(&g_solver));
    if (!g_blas) RP_BLAS(cublasCreate(&g_blas));
    RP_SOLVER(cusolverDnSetStream(g_solver, st));
    RP_BLAS(cublasSetStream(g_blas, st));
}

void dense_handles_release() {
    if (g_solver) cusolverDnDestroy(g_solver);
    if (g_blas) cublasDestroy(g_blas);
    g_solver = nullptr;
    g_blas = nullptr;
}

void dense_build(DenseSystem &d, int len, int dtype, const uint64_t *bits, const double *coeff,
                 int64_t nterms, cudaStream_t st) {
    RP_REQUIRE(len >= 1 && len <= 15, -2, "exact diagonalisation takes 1 to 15 qubits");
    RP_REQUIRE(dtype == 1 || dtype == 2, -2, "dtype must be RP_C64 (1) or RP_C128 (2)");
    RP_REQUIRE(nterms >= 0 && (nterms == 0 || (bits && coeff)), -2, "null term table");
    d.len = len;
    d.dtype = dtype;
    d.dim = 1ull << len;
    const uint64_t dim = d.dim;
    std::vector<DenseTerm> terms;
    for (int64_t k = 0; k < nterms; k++) {
        DenseTerm t{};
        for (int i = 0; i < len; i++) {
            t.x |= ((bits[k] >> (2 * i)) & 1ull) << i;
            t.z |= ((bits[k] >> (2 * i + 1)) & 1ull) << i;
        }
        t.cr = coeff[2 * k];
        t.ci = coeff[2 * k + 1];
        terms.push_back(t);
    }
    ensure_handles(st);
    const size_t mbytes = dim * dim * esz(dtype);
    DenseTerm *dterms = nullptr;
    int *info = nullptr;
    void *work = nullptr;
    try {
        RP_CUDA(cudaMalloc(&d.evecs, mbytes));
        RP_CUDA(cudaMalloc(&d.evals_dev, dim * sizeof(double)));
        RP_CUDA(cudaMalloc((void **)&dterms, std::max<size_t>(1, terms.size()) * sizeof(DenseTerm)));
        RP_CUDA(cudaMalloc((void **)&info, sizeof(int)));
        if (!terms.empty())
            RP_CUDA(cudaMemcpyAsync(dterms, terms.data(), terms.size() * sizeof(DenseTerm),
                                    cudaMemcpyHostToDevice, st));
        RP_CUDA(cudaMemsetAsync(d.evecs, 0, mbytes, st));
        const unsigned nb = (unsigned)((dim + 127) / 128);
        if (dtype == 2)
            k_dense_build<double><<<nb, 128, 0, st>>>(static_cast<Cplx<double> *>(d.evecs), dim, dterms,
                                                      (int)terms.size());
        else
            k_dense_build<float><<<nb, 128, 0, st>>>(static_cast<Cplx<float> *>(d.evecs), dim, dterms,
                                                     (int)terms.size());
        RP_CUDA(cudaGetLastError());
        // eigenvalues into the first dim Reals of evals_dev, eigenvectors in place
        const int n = (int)dim;
        int lwork = 0;
        if (dtype == 2) {
            RP_SOLVER(cusolverDnZheevd_bufferSize(g_solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                                  n, static_cast<cuDoubleComplex *>(d.evecs), n,
                                                  d.evals_dev, &lwork));
            RP_CUDA(cudaMalloc(&work, std::max(1, lwork) * sizeof(cuDoubleComplex)));
            RP_SOLVER(cusolverDnZheevd(g_solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n,
                                       static_cast<cuDoubleComplex *>(d.evecs), n, d.evals_dev,
                                       static_cast<cuDoubleComplex *>(work), lwork, info));
        } else {
            float *w = reinterpret_cast<float *>(d.evals_dev);
            RP_SOLVER(cusolverDnCheevd_bufferSize(g_solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                                  n, static_cast<cuComplex *>(d.evecs), n, w, &lwork));
            RP_CUDA(cudaMalloc(&work, std::max(1, lwork) * sizeof(cuComplex)));
            RP_SOLVER(cusolverDnCheevd(g_solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n,
                                       static_cast<cuComplex *>(d.evecs), n, w,
                                       static_cast<cuComplex *>(work), lwork, info));
        }
        int hinfo = 0;
        RP_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
        d.evals.resize(dim);
        if (dtype == 2) {
            RP_CUDA(cudaMemcpyAsync(d.evals.data(), d.evals_dev, dim * sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
            RP_CUDA(cudaStreamSynchronize(st));
        } else {
            std::vector<float> wf(dim);
            RP_CUDA(cudaMemcpyAsync(wf.data(), d.evals_dev, dim * sizeof(float), cudaMemcpyDeviceToHost, st));
            RP_CUDA(cudaStreamSynchronize(st));
            for (uint64_t i = 0; i < dim; i++) d.evals[i] = wf[i];
        }
        RP_REQUIRE(hinfo == 0, -3, "the eigensolver (heevd) failed, info " + std::to_string(hinfo));
    } catch (...) {
        cudaFree(dterms);
        cudaFree(info);
        cudaFree(work);
        dense_free(d);
        throw;
    }
    cudaFree(dterms);
    cudaFree(info);
    cudaFree(work);
}

void dense_free(DenseSystem &d) {
    if (d.evecs) cudaFree(d.evecs);
    if (d.evals_dev) cudaFree(d.evals_dev);
    d.evecs = nullptr;
    d.evals_dev = nullptr;
    d.evals.clear();
}

void dense_expm(const DenseSystem &d, double cr, double ci, void *out, cudaStream_t st) {
    RP_REQUIRE(d.evecs, -2, "empty eigensystem");
    const uint64_t dim = d.dim;
    const size_t mbytes = dim * dim * esz(d.dtype);
    ensure_handles(st);
    void *tmp = scratch_get(SCR_EXPM_DENSE, mbytes, st);
    const unsigned nb = (unsigned)std::min<uint64_t>((dim * dim + 255) / 256, 8u * num_sms());
    const int n = (int)dim;
    if (d.dtype == 2) {
        k_scale_cols<double><<<nb, 256, 0, st>>>(static_cast<Cplx<double> *>(tmp),
                                                 static_cast<const Cplx<double> *>(d.evecs),
                                                 d.evals_dev, dim, cr, ci);
        RP_CUDA(cudaGetLastError());
        const cuDoubleComplex one{1.0, 0.0}, zero{0.0, 0.0};
        RP_BLAS(cublasZgemm(g_blas, CUBLAS_OP_N, CUBLAS_OP_C, n, n, n, &one,
                            static_cast<const cuDoubleComplex *>(tmp), n,
                            static_cast<const cuDoubleComplex *>(d.evecs), n, &zero,
                            static_cast<cuDoubleComplex *>(out), n));
    } else {
        k_scale_cols<float><<<nb, 256, 0, st>>>(static_cast<Cplx<float> *>(tmp),
                                                static_cast<const Cplx<float> *>(d.evecs),
                                                reinterpret_cast<const float *>(d.evals_dev), dim, cr, ci);
        RP_CUDA(cudaGetLastError());
        const cuComplex one{1.f, 0.f}, zero{0.f, 0.f};
        RP_BLAS(cublasCgemm(g_blas, CUBLAS_OP_N, CUBLAS_OP_C, n, n, n, &one,
                            static_cast<const cuComplex *>(tmp), n, static_cast<const cuComplex *>(d.evecs),
                            n, &zero, static_cast<cuComplex *>(out), n));
    }
}

void dense_column(const DenseSystem &d, int64_t col, void *out, cudaStream_t st) {
    RP_REQUIRE(d.evecs, -2, "empty eigensystem");
    RP_REQUIRE(col >= 0 && (uint64_t)col < d.dim, -2, "eigenvector index out of range");
    const size_t vb = d.dim * esz(d.dtype);
    RP_CUDA(cudaMemcpyAsync(out, static_cast<const char *>(d.evecs) + (size_t)col * vb, vb,
                            cudaMemcpyDeviceToDevice, st));
}

}  // namespace rp
