// ref_io.h -- term-file reading and SpinOp construction shared by the
// reference drivers (ref_driver.cc, ref_gpu_driver.cc).  TEST INFRASTRUCTURE
// ONLY.  Include after <reapers.h> with `using namespace REAPERS` in effect.
//
// Term file (little endian): int64 T, int32 len, then T records
// {u64 bits, f64 re, f64 im}; the coefficient is the stored one (sigma_y's i
// folded in, inc/ops.h:285-288).
#pragma once

#include <complex>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

struct Term { uint64_t bits; double re, im; };

static std::vector<Term> read_terms(const char *path, int &len) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { std::cerr << "cannot open " << path << "\n"; exit(2); }
    int64_t T; int32_t l;
    f.read((char *)&T, 8); f.read((char *)&l, 4);
    std::vector<Term> t(T);
    f.read((char *)t.data(), T * sizeof(Term));
    len = l;
    return t;
}

// Build a SpinOp with the given internal bits and stored coefficient through
// the public API: right-multiply single-site sigma matrices (no carry-over
// sign arises between different sites), then fix the coefficient.
template <typename Fp>
static SpinOp<Fp> make_op(const Term &t) {
    auto op = SpinOp<Fp>::identity();
    for (int i = 0; i < 32; i++) {
        unsigned s = (t.bits >> (2 * i)) & 3;
        if (s == 1) op *= SpinOp<Fp>::sigma_x(i);
        else if (s == 2) op *= SpinOp<Fp>::sigma_z(i);
        else if (s == 3) op *= SpinOp<Fp>::sigma_y(i);
    }
    // the coefficient is now i^ny; multiply by target * conj(i^ny) (exact)
    int ny = 0;
    for (int i = 0; i < 32; i++) if (((t.bits >> (2 * i)) & 3) == 3) ny++;
    std::complex<double> cur(1, 0);
    for (int k = 0; k < (ny & 3); k++) cur *= std::complex<double>(0, 1);
    std::complex<double> f = std::complex<double>(t.re, t.im) * std::conj(cur);
    op *= complex<Fp>((Fp)f.real(), (Fp)f.imag());
    return op;
}

