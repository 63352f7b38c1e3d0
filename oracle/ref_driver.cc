// ref_driver.cc -- runs the REAPERS reference library itself (its headers,
// compiled unmodified from the reference checkout with REAPERS_NOGPU and the
// default (float) precision, as examples/syk.cc is, against the project-written
// Eigen subset in eigen_shim/).
//
// TEST INFRASTRUCTURE ONLY: it makes golden fixtures, pins the C restatement
// in rp_oracle.c, and is the timed CPU baseline (the reference's own
// OpenMP CPUImpl).  The product never links or calls it.  Built by
// oracle/Makefile into oracle/_ref/ref_driver.
//
// File formats (little endian):
//   terms : int64 T, int32 len, then T records {u64 bits, f64 re, f64 im}
//   vector: int64 D, then D records {f64 re, f64 im}
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <vector>

#include <omp.h>

#define REAPERS_NOGPU

#include <reapers.h>

using namespace REAPERS;
using namespace REAPERS::Model;
using namespace REAPERS::EvolutionAlgorithm;

#include "ref_io.h"

// CPUImpl with call counters, so that the number of H.psi products and inner
// products of a reference evolve can be compared with the oracle's.
struct CountingImpl : CPUImpl {
    static inline long n_apply = 0;
    static inline long n_prod = 0;
    template <RealScalar FpType>
    static void apply_ops(typename SpinOp<FpType>::IndexType len, BufType<FpType> res,
                          const HostSumOps<FpType> &ops, ConstBufType<FpType> vec) {
        n_apply++;
        CPUImpl::apply_ops(len, res, ops, vec);
    }
    template <RealScalar FpType>
    static complex<FpType> vec_prod(VecSizeType<FpType> size, ConstBufType<FpType> v0,
                                    ConstBufType<FpType> v1) {
        n_prod++;
        return CPUImpl::vec_prod(size, v0, v1);
    }
    template <RealScalar FpType>
    static FpType vec_norm(VecSizeType<FpType> size, ConstBufType<FpType> v0) {
        return std::sqrt(vec_prod(size, v0, v0).real());
    }
};

using Ops = HostSumOps<double>;
using St = State<double, CountingImpl>;

static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static void write_records(std::ofstream &f, const Ops &ops) {
    for (auto &op : ops) {
        // SpinOp keeps its stored coefficient private; coefficient() returns
        // it times (-i)^(number of sigma_y factors mod 4) (ops.h:343-355), so
        // multiply that factor back out (multiplication by i is exact).
        Term t;
        t.bits = op.get_bit_string();
        auto c = op.coefficient();
        int ny = 0;
        for (int i = 0; i < 32; i++) if (((t.bits >> (2 * i)) & 3) == 3) ny++;
        std::complex<double> cc(c.real(), c.imag());
        for (int k = 0; k < (ny & 3); k++) cc *= std::complex<double>(0, 1);
        t.re = cc.real(); t.im = cc.imag();
        f.write((const char *)&t, sizeof t);
    }
}

static void write_terms(const char *path, const Ops &ops, int len) {
    std::ofstream f(path, std::ios::binary);
    int64_t T = ops.size(); int32_t l = len;
    f.write((const char *)&T, 8); f.write((const char *)&l, 4);
    write_records(f, ops);
}

template <typename Fp = double>
static HostSumOps<Fp> build_ops(const std::vector<Term> &terms) {
    HostSumOps<Fp> ops;
    for (auto &t : terms) ops += make_op<Fp>(t);
    return ops;
}

// Time the body of CPUImpl::apply_ops (inc/cpuimpl.h:747-753) -- the
// reference's SpinOp::apply per (row, term), terms in list order -- over the
// bounded slice of output rows [row0, row0 + nrows) of a 2^len state, with
// OpenMP over rows as the reference does.  Prints seconds per slice.
template <typename Fp>
static int bench_rows(const std::vector<Term> &terms, int len, uint64_t row0, uint64_t nrows,
                      int reps) {
    auto ops = build_ops<Fp>(terms);
    const uint64_t D = 1ull << len;
    std::vector<complex<Fp>> vec(D), res(nrows);
    std::mt19937_64 g(12345);
    std::normal_distribution<double> nd;
    for (auto &v : vec) v = complex<Fp>((Fp)nd(g), (Fp)nd(g));
    double best = 1e300;
    for (int r = 0; r < reps; r++) {
        double t0 = now();
        #pragma omp parallel for schedule(static)
        for (uint64_t i = 0; i < nrows; i++) {
            complex<Fp> acc = 0;
            for (const auto &op : ops) {
                typename SpinOp<Fp>::StateType n = 0;
                auto coeff = op.apply((typename SpinOp<Fp>::StateType)(row0 + i), n);
                acc += coeff * vec[n];
            }
            res[i] = acc;
        }
        best = std::min(best, now() - t0);
    }
    double chk = 0;
    for (auto &v : res) chk += std::abs(v);
    printf("{\"seconds\": %.6e, \"rows\": %llu, \"len\": %d, \"terms\": %zu, \"threads\": %d, \"check\": %.6e}\n",
           best, (unsigned long long)nrows, len, ops.size(), omp_get_max_threads(), chk);
    return 0;
}

static std::vector<std::complex<double>> read_vec(const char *path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { std::cerr << "cannot open " << path << "\n"; exit(2); }
    int64_t D; f.read((char *)&D, 8);
    std::vector<std::complex<double>> v(D);
    f.read((char *)v.data(), D * 16);
    return v;
}

static void write_vec(const char *path, const std::vector<std::complex<double>> &v) {
    std::ofstream f(path, std::ios::binary);
    int64_t D = v.size();
    f.write((const char *)&D, 8);
    f.write((const char *)v.data(), D * 16);
}

static void load_state(St &s, const std::vector<std::complex<double>> &v) {
    for (size_t i = 0; i < v.size(); i++) s[i] = complex<double>(v[i].real(), v[i].imag());
}

static std::vector<std::complex<double>> dump_state(const St &s) {
    std::vector<std::complex<double>> v(s.dim());
    for (size_t i = 0; i < v.size(); i++) { auto c = s[i]; v[i] = {c.real(), c.imag()}; }
    return v;
}


int main(int argc, char **argv) {
    if (argc < 2) { std::cerr << "usage: ref_driver MODE ...\n"; return 1; }
    std::string mode = argv[1];
    if (mode == "syk") {
        // syk N sp J seed out  -- SYK::gen_ham with std::mt19937(seed), non-block form
        int N = atoi(argv[2]); double sp = atof(argv[3]), J = atof(argv[4]);
        unsigned seed = (unsigned)strtoul(argv[5], 0, 10);
        std::mt19937 rg(seed);
        SYK<double, CPUImpl, FermionOpNonBlockForm> syk(N, sp, J);
        auto ham = syk.gen_ham(rg);
        write_terms(argv[6], ham, N / 2);
        return 0;
    }
    if (mode == "majorana") {
        // majorana N out  -- all N non-block Majorana strings b_0..b_{N-1}
        int N = atoi(argv[2]);
        SYK<double, CPUImpl, FermionOpNonBlockForm> syk(N, 0.0, 1.0);
        std::ofstream f(argv[3], std::ios::binary);
        int64_t T = N; int32_t l = N / 2;
        f.write((const char *)&T, 8); f.write((const char *)&l, 4);
        for (int n = 0; n < N; n++) write_records(f, Ops(syk.fermion_ops(n)));
        return 0;
    }
    if (mode == "majorana_block") {
        // majorana_block N out -- the parity-block Majoranas b_n = [[0, LR], [RL, 0]]
        // of FermionOpBlockForm (inc/fermions.h:308-366) on N/2-1 qubits:
        // records LR_0, RL_0, LR_1, RL_1, ...
        int N = atoi(argv[2]);
        SYK<double, CPUImpl, FermionOpBlockForm> syk(N, 0.0, 1.0);
        std::ofstream f(argv[3], std::ios::binary);
        int64_t T = 2 * N; int32_t l = N / 2 - 1;
        f.write((const char *)&T, 8); f.write((const char *)&l, 4);
        for (int n = 0; n < N; n++) {
            write_records(f, Ops(syk.fermion_ops(n).LR));
            write_records(f, Ops(syk.fermion_ops(n).RL));
        }
        return 0;
    }
    if (mode == "syk_block") {
        // syk_block N sp J seed outLL outRR -- SYK::gen_ham with std::mt19937(seed)
        // in parity-block form: the blocks H_LL and H_RR on N/2-1 qubits
        int N = atoi(argv[2]); double sp = atof(argv[3]), J = atof(argv[4]);
        unsigned seed = (unsigned)strtoul(argv[5], 0, 10);
        std::mt19937 rg(seed);
        SYK<double, CPUImpl, FermionOpBlockForm> syk(N, sp, J);
        auto ham = syk.gen_ham(rg);
        write_terms(argv[6], Ops(ham.LL), N / 2 - 1);
        write_terms(argv[7], Ops(ham.RR), N / 2 - 1);
        return 0;
    }
    if (mode == "otoc_block") {
        // otoc_block termsLL termsRR opterm psi0 out krydim tol t1 t2 ...
        //   OTOC::evolve of examples/syk.cc:270-283 at beta = 0 on one parity
        //   block: s = op s; e^{-iH_RR t}; e^{+iH_LL t}; op; e^{-iH_RR t};
        //   e^{+iH_LL t}; F = <psi0|s>
        int len, lo;
        auto LL = build_ops(read_terms(argv[2], len));
        auto RR = build_ops(read_terms(argv[3], len));
        auto op = build_ops(read_terms(argv[4], lo));
        auto v = read_vec(argv[5]);
        int krydim = atoi(argv[7]);
        double tol = atof(argv[8]);
        St init(len), s(len);
        load_state(init, v);
        std::ofstream f(argv[6], std::ios::binary);
        int64_t npts = argc - 9;
        f.write((const char *)&npts, 8);
        for (int a = 9; a < argc; a++) {
            double t = atof(argv[a]);
            s = init;
            s *= op;
            s.evolve(RR, t, 0.0, krydim, tol);
            s.evolve(LL, -t, 0.0, krydim, tol);
            s *= op;
            s.evolve(RR, t, 0.0, krydim, tol);
            s.evolve(LL, -t, 0.0, krydim, tol);
            auto c = init * s;
            double re = c.real(), im = c.imag();
            f.write((const char *)&re, 8);
            f.write((const char *)&im, 8);
        }
        return 0;
    }
    if (mode == "roundtrip") {
        // roundtrip terms out -- terms through SpinOp/HostSumOps and back
        int len; auto terms = read_terms(argv[2], len);
        write_terms(argv[3], build_ops(terms), len);
        return 0;
    }
    if (mode == "apply") {
        // apply terms in out  -- (ops * State), State::operator* (state.h:335-343)
        int len; auto terms = read_terms(argv[2], len);
        auto ops = build_ops(terms);
        auto v = read_vec(argv[3]);
        St s(len);
        load_state(s, v);
        St r = ops * s;
        write_vec(argv[4], dump_state(r));
        return 0;
    }
    if (mode == "evolve") {
        // evolve terms in out t beta krydim tol max_iters
        int len; auto terms = read_terms(argv[2], len);
        auto ops = build_ops(terms);
        auto v = read_vec(argv[3]);
        double t = atof(argv[5]), beta = atof(argv[6]), tol = atof(argv[8]);
        int krydim = atoi(argv[7]), max_iters = atoi(argv[9]);
        St s(len);
        load_state(s, v);
        CountingImpl::n_apply = CountingImpl::n_prod = 0;
        double t0 = now();
        s.evolve(ops, t, beta, krydim, tol, max_iters);
        double t1 = now();
        write_vec(argv[4], dump_state(s));
        printf("{\"applies\": %ld, \"prods\": %ld, \"seconds\": %.6f}\n",
               CountingImpl::n_apply, CountingImpl::n_prod, t1 - t0);
        return 0;
    }
    if (mode == "otoc") {
        // otoc terms wterm vterm psi0 out krydim tol t1 t2 ...
        //   the sequence of examples/simple-syk-krylov.cc:42-57 at beta = 0:
        //   psi = V psi0; e^{-iHt}; W; e^{iHt}; V; e^{-iHt}; W; e^{iHt}; <psi0|psi>
        int len; auto terms = read_terms(argv[2], len);
        int lw, lv;
        auto W = build_ops(read_terms(argv[3], lw));
        auto V = build_ops(read_terms(argv[4], lv));
        auto ops = build_ops(terms);
        auto v = read_vec(argv[5]);
        int krydim = atoi(argv[7]);
        double tol = atof(argv[8]);
        St init(len), psi(len);
        load_state(init, v);
        std::ofstream f(argv[6], std::ios::binary);
        int64_t npts = argc - 9;
        f.write((const char *)&npts, 8);
        CountingImpl::n_apply = 0;
        double t0 = now();
        for (int a = 9; a < argc; a++) {
            double t = atof(argv[a]);
            psi = init;
            psi *= V;
            psi.evolve(ops, t, 0.0, krydim, tol);
            psi *= W;
            psi.evolve(ops, -t, 0.0, krydim, tol);
            psi *= V;
            psi.evolve(ops, t, 0.0, krydim, tol);
            psi *= W;
            psi.evolve(ops, -t, 0.0, krydim, tol);
            auto c = init * psi;
            double re = c.real(), im = c.imag();
            f.write((const char *)&re, 8);
            f.write((const char *)&im, 8);
        }
        printf("{\"applies\": %ld, \"seconds\": %.6f}\n", CountingImpl::n_apply, now() - t0);
        return 0;
    }
    if (mode == "bench_apply") {
        // bench_apply terms reps  -- time State::operator*= (zero_vec + apply_ops)
        // on a random state; prints seconds per H.psi
        int len; auto terms = read_terms(argv[2], len);
        int reps = atoi(argv[3]);
        auto ops = build_ops(terms);
        St s(len);
        s.random_state();
        s *= ops;   // warm-up (and the dense-matrix build when #terms >= 2^len)
        double t0 = now();
        for (int r = 0; r < reps; r++) s *= ops;
        double dt = (now() - t0) / reps;
        printf("{\"seconds_per_apply\": %.6e, \"len\": %d, \"terms\": %zu}\n", dt, len, ops.size());
        return 0;
    }
    if (mode == "bench_rows") {
        // bench_rows terms fp(32|64) row0 nrows reps
        int len; auto terms = read_terms(argv[2], len);
        int fp = atoi(argv[3]);
        uint64_t row0 = strtoull(argv[4], 0, 10), nrows = strtoull(argv[5], 0, 10);
        int reps = atoi(argv[6]);
        if (row0 + nrows > (1ull << len)) { std::cerr << "row slice out of range\n"; return 1; }
        return fp == 32 ? bench_rows<float>(terms, len, row0, nrows, reps)
                        : bench_rows<double>(terms, len, row0, nrows, reps);
    }
    std::cerr << "unknown mode " << mode << "\n";
    return 1;
}
