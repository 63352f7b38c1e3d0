// Exact diagonalisation on the device (the reference's dense GPU path).
#pragma once

#include <vector>

#include "rp_common.cuh"

namespace rp {

// One Pauli term: X and Z masks (bit i = qubit i) and its stored coefficient.
struct DenseTerm {
    uint64_t x = 0, z = 0;
    double cr = 0, ci = 0;
};

// The eigensystem of a Hermitian Pauli sum on 2^len states: eigenvectors as
// the columns of a dim x dim column-major device matrix in the Hamiltonian's
// precision, eigenvalues ascending (device, that precision; host, FP64).
struct DenseSystem {
    int len = 0, dtype = 0;
    uint64_t dim = 0;
    void *evecs = nullptr;
    double *evals_dev = nullptr;
    std::vector<double> evals;
};

void dense_build(DenseSystem &d, int len, int dtype, const uint64_t *bits, const double *coeff,
                 int64_t nterms, cudaStream_t st);
void dense_free(DenseSystem &d);
// out (dim x dim, column-major, device) = exp((cr + i ci) H)
void dense_expm(const DenseSystem &d, double cr, double ci, void *out, cudaStream_t st);
// out (device vector) = eigenvector col
void dense_column(const DenseSystem &d, int64_t col, void *out, cudaStream_t st);
// res = M v for a dense dim x dim column-major device matrix M
void dense_matvec(int dtype, uint64_t dim, const void *M, const void *v, void *res, cudaStream_t st);
void dense_handles_release();

int num_sms();

}  // namespace rp
