// ref_gpu_driver.cc -- the REAPERS reference's own GPU backend (GPUImpl with
// its krnl_apply_ops kernel, src/krnl.cu:81-94, launched by
// GPUImpl::apply_ops, src/krnl.cu:220-257), compiled unmodified from the
// reference checkout for sm_100a together with its src/krnl.cu, against the
// project-written Eigen subset in eigen_shim/.
//
// TEST INFRASTRUCTURE ONLY: a second, GPU-side baseline beside the reference's
// CPU build.  It times the reference's one-thread-per-element H.psi kernel on
// the same B200 and workload as the product's row kernel, and writes its
// output for a parity check.  The product never links or calls it.  Built by
// oracle/Makefile into oracle/_ref/ref_gpu_driver where the reference checkout
// exists.
//
// usage:
//   ref_gpu_driver apply terms fp vec out   H.psi of a vector (file formats of
//                                           ref_driver.cc), fp = 32 or 64
//   ref_gpu_driver bench terms fp reps      ms per GPUImpl::apply_ops on a
//                                           random state (CUDA events, after one
//                                           warm-up apply), as JSON
//   ref_gpu_driver evolve terms fp t krydim tol
//                                           the reference's restarted Krylov
//                                           (State::evolve, inc/algo.h:267-365)
//                                           on its GPU backend from a random
//                                           state: seconds and H.psi count, JSON
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <reapers.h>

using namespace REAPERS;

#include "ref_io.h"

// GPUImpl with an H.psi counter, as ref_driver.cc's CountingImpl does for
// the CPU backend.
struct CountingGPU : GPUImpl {
    static inline long n_apply = 0;
    template <RealScalar FpType>
    static void apply_ops(typename SpinOp<FpType>::IndexType len, BufType<FpType> res,
                          const DevSumOps<FpType> &ops, ConstBufType<FpType> vec) {
        n_apply++;
        GPUImpl::apply_ops(len, res, ops, vec);
    }
};

// the reference's GPU Hamiltonian (DevSumOps) from the stored terms
template <typename Fp>
static typename GPUImpl::template SumOps<Fp> build_ops(const std::vector<Term> &terms) {
    HostSumOps<Fp> h;
    for (const auto &t : terms) h += make_op<Fp>(t);
    return typename GPUImpl::template SumOps<Fp>(h);
}

template <typename Fp>
static int run(int argc, char **argv, const std::string &mode, const std::vector<Term> &terms,
               int len) {
    using GSt = State<Fp, GPUImpl>;
    using CSt = State<Fp, CPUImpl>;
    const auto ops = build_ops<Fp>(terms);
    if (mode == "apply") {
        std::ifstream f(argv[4], std::ios::binary);
        int64_t D = 0;
        f.read((char *)&D, 8);
        std::vector<std::complex<double>> v(D);
        f.read((char *)v.data(), D * 16);
        CSt c(len);
        for (int64_t i = 0; i < D; i++) c[i] = complex<Fp>((Fp)v[i].real(), (Fp)v[i].imag());
        GSt g(c);
        GSt r = ops * g;
        CSt rh(r);
        std::ofstream o(argv[5], std::ios::binary);
        o.write((const char *)&D, 8);
        for (int64_t i = 0; i < D; i++) {
            const complex<Fp> z = rh[i];
            const double re = z.real(), im = z.imag();
            o.write((const char *)&re, 8);
            o.write((const char *)&im, 8);
        }
        return 0;
    }
    if (mode == "evolve") {
        const double t = std::atof(argv[4]);
        const int krydim = std::atoi(argv[5]);
        const double tol = std::atof(argv[6]);
        State<Fp, CountingGPU> x(len);
        x.random_state();
        State<Fp, CountingGPU> w(x);
        w.evolve(ops, 0.01, 0.0, krydim, (Fp)tol);   // warm-up: uploads, buffers
        CountingGPU::n_apply = 0;
        cudaDeviceSynchronize();
        const auto t0 = std::chrono::steady_clock::now();
        x.evolve(ops, t, 0.0, krydim, (Fp)tol);
        cudaDeviceSynchronize();
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("{\"seconds\": %.4f, \"applies\": %ld, \"len\": %d, \"fp\": %d}\n", sec,
                    CountingGPU::n_apply, len, (int)(8 * sizeof(Fp)));
        return 0;
    }
    const int reps = std::atoi(argv[4]);
    GSt x(len), y(len);
    x.random_state();
    y.zero_state();
    GPUImpl::apply_ops(len, y.buf(), ops, x.buf());   // warm-up: uploads the terms
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    for (int i = 0; i < reps; i++) GPUImpl::apply_ops(len, y.buf(), ops, x.buf());
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    std::printf("{\"ms_per_apply\": %.4f, \"reps\": %d, \"terms\": %zu, \"len\": %d, \"fp\": %d}\n",
                ms / reps, reps, ops.size(), len, (int)(8 * sizeof(Fp)));
    return 0;
}

int main(int argc, char **argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: ref_gpu_driver apply|bench|evolve terms fp ...\n");
        return 1;
    }
    const std::string mode = argv[1];
    int len = 0;
    const auto terms = read_terms(argv[2], len);
    const int fp = std::atoi(argv[3]);
    if (mode != "apply" && mode != "bench" && mode != "evolve") return 1;
    return fp == 64 ? run<double>(argc, argv, mode, terms, len) : run<float>(argc, argv, mode, terms, len);
}
