// dropin_driver.cc -- the reference library's own host code (State, Krylov,
// SYK, FermionOpNonBlockForm; its headers compiled unmodified from the
// reference checkout with REAPERS_NOGPU against eigen_shim/) run twice in one
// process: on its CPU backend (CPUImpl) and on B200Impl
// (include/rpb200_impl.hpp, i.e. librpb200's sm_100a kernels).
//
// TEST INFRASTRUCTURE ONLY: it shows that B200Impl is a drop-in backend for
// the reference's unchanged algorithms and measures the difference of every
// result against the CPU backend.  Built by oracle/Makefile into
// oracle/_ref/dropin_driver; run by tests/test_gpu_dropin.py.
//
// usage: dropin_driver N sparsity seed t krydim
// prints one JSON object of relative differences (GPU backend vs CPU backend)
// and both backends' ground-state energies.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>

#define REAPERS_NOGPU

#include <reapers.h>

#include "rpb200_impl.hpp"

using namespace REAPERS;
using namespace REAPERS::Model;
using namespace REAPERS::EvolutionAlgorithm;

using CSt = State<double, CPUImpl>;
using GSt = State<double, B200Impl>;

// ||a - b|| / ||b|| with a moved to the host backend
static double rel_diff(const GSt &g, const CSt &c) {
    CSt gh(g);
    double num = 0, den = 0;
    for (size_t i = 0; i < c.dim(); i++) {
        auto d = gh[i] - c[i];
        num += std::norm(std::complex<double>(d.real(), d.imag()));
        auto v = c[i];
        den += std::norm(std::complex<double>(v.real(), v.imag()));
    }
    return std::sqrt(num / den);
}

template <typename Ops>
static double term_diff(const Ops &a, const HostSumOps<double> &b) {
    if (a.size() != b.size()) return 1e300;
    double d = 0;
    auto ib = b.begin();
    for (auto ia = a.begin(); ia != a.end(); ++ia, ++ib) {
        if (ia->get_bit_string() != ib->get_bit_string()) return 1e300;
        d = std::max(d, (double)std::abs(ia->coefficient() - ib->coefficient()));
    }
    return d;
}

int main(int argc, char **argv) {
    if (argc < 6) {
        std::fprintf(stderr, "usage: dropin_driver N sparsity seed t krydim\n");
        return 1;
    }
    const int N = std::atoi(argv[1]);
    const double sp = std::atof(argv[2]);
    const unsigned seed = (unsigned)std::strtoul(argv[3], nullptr, 10);
    const double t = std::atof(argv[4]);
    const int krydim = std::atoi(argv[5]);
    const int L = N / 2;
    const double tol = 1e-14;

    // the same model and generator on both backends (inc/syk.h:239-263)
    SYK<double, CPUImpl, FermionOpNonBlockForm> syk_c(N, sp, 1.0);
    SYK<double, B200Impl, FermionOpNonBlockForm> syk_g(N, sp, 1.0);
    std::mt19937 rg_c(seed), rg_g(seed);
    HostSumOps<double> ham_c = syk_c.gen_ham(rg_c);
    B200SumOps<double> ham_g = syk_g.gen_ham(rg_g);
    const double terms = term_diff(ham_g, ham_c);

    // one random state, moved to the device by State's conversion constructor
    CSt c0(L);
    {
        std::mt19937 rs(seed + 1);
        std::normal_distribution<double> nd(0.0, 1.0);
        for (size_t i = 0; i < c0.dim(); i++) c0[i] = complex<double>(nd(rs), nd(rs));
        c0 *= 1.0 / c0.norm();
    }
    GSt g0(c0);
    const double roundtrip = rel_diff(g0, c0);
    // element access through the device proxy
    complex<double> e3 = g0[3];
    const double elem = std::abs(e3 - c0[3]);

    // H psi: State operator* (inc/state.h:335-343)
    CSt c1 = ham_c * c0;
    GSt g1 = ham_g * g0;
    const double apply = rel_diff(g1, c1);

    // the reference's own restarted Krylov (inc/algo.h:267-365) on both backends
    CSt c2(c0);
    GSt g2(g0);
    c2.evolve(ham_c, t, 0.0, krydim, tol);
    g2.evolve(ham_g, t, 0.0, krydim, tol);
    const double evolve = rel_diff(g2, c2);

    // the GPU-resident Krylov through the same State call
    GSt g3(g0);
    g3.evolve<B200Krylov>(ham_g, t, 0.0, krydim, tol);
    const double evolve_fused = rel_diff(g3, c2);

    // imaginary time as well: exp(-(beta + i t) H)
    CSt c4(c0);
    GSt g4(g0);
    c4.evolve(ham_c, 0.3 * t, 0.2, krydim, tol);
    g4.evolve<B200Krylov>(ham_g, 0.3 * t, 0.2, krydim, tol);
    const double evolve_beta = rel_diff(g4, c4);

    // OTOC sequence of examples/simple-syk-krylov.cc:42-57 with W = b_{N-1}, V = b_{N-2}
    HostSumOps<double> Wc(syk_c.fermion_ops(N - 1)), Vc(syk_c.fermion_ops(N - 2));
    B200SumOps<double> Wg(syk_g.fermion_ops(N - 1)), Vg(syk_g.fermion_ops(N - 2));
    CSt pc(c0);
    GSt pg(g0);
    pc *= Vc;
    pg *= Vg;
    pc.evolve(ham_c, t, 0.0, krydim, tol);
    pg.evolve<B200Krylov>(ham_g, t, 0.0, krydim, tol);
    pc *= Wc;
    pg *= Wg;
    pc.evolve(ham_c, -t, 0.0, krydim, tol);
    pg.evolve<B200Krylov>(ham_g, -t, 0.0, krydim, tol);
    pc *= Vc;
    pg *= Vg;
    pc.evolve(ham_c, t, 0.0, krydim, tol);
    pg.evolve<B200Krylov>(ham_g, t, 0.0, krydim, tol);
    pc *= Wc;
    pg *= Wg;
    pc.evolve(ham_c, -t, 0.0, krydim, tol);
    pg.evolve<B200Krylov>(ham_g, -t, 0.0, krydim, tol);
    const auto Fc = c0 * pc;
    const auto Fg = g0 * pg;
    const double otoc = std::abs(Fg - Fc) / std::abs(c0 * c0);

    // a moved operator keeps no device table of its old term list: apply
    // one, move-assign another onto it, apply again
    double moved = 0.0;
    {
        B200SumOps<double> a(ham_g), b(SpinOp<double>::sigma_z(0));
        GSt t1 = a * g0;
        (void)t1;
        a = std::move(b);
        GSt t2 = a * g0;
        CSt z0(c0);
        z0 *= HostSumOps<double>(SpinOp<double>::sigma_z(0));
        moved = rel_diff(t2, z0);
    }

    // changing the operator drops its device table (release()); the next
    // apply uploads the new term list
    ham_c += SpinOp<double>::sigma_x(0) * SpinOp<double>::sigma_y(1);
    ham_g += SpinOp<double>::sigma_x(0) * SpinOp<double>::sigma_y(1);
    CSt c5 = ham_c * c0;
    GSt g5 = ham_g * g0;
    const double mutate = rel_diff(g5, c5);

    // the reference's ground-state Lanczos (inc/algo.h:180-257) on both
    // backends; the random starting states differ, the answers must not
    CSt gc(L);
    GSt gg(L);
    const double Ec = gc.ground_state(ham_c, 20, 1e-10, 400);
    const double Eg = gg.ground_state(ham_g, 20, 1e-10, 400);
    CSt ggh(gg);
    const double overlap = std::abs(gc * ggh);

    // exact diagonalisation (inc/algo.h:29-54) on both backends: B200Impl's
    // eigensystem, matexp and mat_mul run on the device (rp_dense_*); the
    // CPU backend's eigen solve (the Eigen-API subset's Jacobi method) runs
    // only up to 2^8 states, above that the references are the CPU backend's
    // Lanczos ground state (gc, above) and restarted Krylov evolve of the
    // current (changed) operator
    CSt cm(c0), cb(c0);
    cm.evolve(ham_c, t, 0.0, krydim, tol);
    cb.evolve(ham_c, 0.3 * t, 0.2, krydim, tol);
    GSt eg(L);
    const double Eed = eg.template ground_state<ExactDiagonalization>(ham_g);
    CSt egh(eg);
    const double ed_overlap = std::abs(gc * egh);
    GSt ee(g0);
    ee.template evolve<ExactDiagonalization>(ham_g, t, 0.0);
    const double ed_evolve = rel_diff(ee, cm);
    GSt ee2(g0);
    ee2.template evolve<ExactDiagonalization>(ham_g, t, 0.0);   // the matexp cache's hit
    const double ed_cached = rel_diff(ee2, cm);
    const double ed_cache_bytes = (double)B200Impl::get_current_cache_size();
    GSt eb(g0);
    eb.template evolve<ExactDiagonalization>(ham_g, 0.3 * t, 0.2);
    const double ed_beta = rel_diff(eb, cb);
    double ed_cpu_energy = 0.0, ed_cpu_evolve = 0.0;
    int ed_cpu = 0;
    if (L <= 8) {
        CSt ec(L);
        ed_cpu_energy = ec.template ground_state<ExactDiagonalization>(ham_c);
        CSt ev(c0);
        ev.template evolve<ExactDiagonalization>(ham_c, t, 0.0);
        ed_cpu_evolve = rel_diff(ee, ev);
        ed_cpu = 1;
    }

    // parity-block form (FermionOpBlockForm, BlockDiag, BlockState): the
    // OTOC of examples/syk.cc (OTOC::evolve at beta = 0) on one block of
    // N/2 - 1 qubits, and a BlockState evolved under BlockDiag(H_LL, H_RR)
    SYK<double, CPUImpl, FermionOpBlockForm> bsyk_c(N, sp, 1.0);
    SYK<double, B200Impl, FermionOpBlockForm> bsyk_g(N, sp, 1.0);
    std::mt19937 brg_c(seed), brg_g(seed);
    auto bham_c = bsyk_c.gen_ham(brg_c);
    auto bham_g = bsyk_g.gen_ham(brg_g);
    const double bterms = std::max(term_diff(bham_g.LL, bham_c.LL), term_diff(bham_g.RR, bham_c.RR));
    CSt b0(L - 1);
    {
        std::mt19937 rs(seed + 2);
        std::normal_distribution<double> nd(0.0, 1.0);
        for (size_t i = 0; i < b0.dim(); i++) b0[i] = complex<double>(nd(rs), nd(rs));
        b0 *= 1.0 / b0.norm();
    }
    GSt bg0(b0);
    const auto &opc = bsyk_c.fermion_ops(N - 2).LR;
    const auto &opg = bsyk_g.fermion_ops(N - 2).LR;
    CSt sc(b0);
    GSt sg(bg0);
    sc *= opc;
    sg *= opg;
    sc.evolve(bham_c.RR, t, 0.0, krydim, tol);
    sg.evolve<B200Krylov>(bham_g.RR, t, 0.0, krydim, tol);
    sc.evolve(bham_c.LL, -t, 0.0, krydim, tol);
    sg.evolve<B200Krylov>(bham_g.LL, -t, 0.0, krydim, tol);
    sc *= opc;
    sg *= opg;
    sc.evolve(bham_c.RR, t, 0.0, krydim, tol);
    sg.evolve(bham_g.RR, t, 0.0, krydim, tol);   // the reference's Krylov on B200Impl
    sc.evolve(bham_c.LL, -t, 0.0, krydim, tol);
    sg.evolve(bham_g.LL, -t, 0.0, krydim, tol);
    const auto Fbc = b0 * sc;
    const auto Fbg = bg0 * sg;
    const double otoc_block = std::abs(Fbg - Fbc) / std::abs(b0 * b0);
    BlockState<double, CPUImpl> bsc(L - 1);
    BlockState<double, B200Impl> bsg(L - 1);
    bsc.L = b0;
    bsc.R = CSt(b0);
    bsc.R *= complex<double>(0.6, -0.8);
    bsg.L = bg0;
    bsg.R = GSt(bg0);
    bsg.R *= complex<double>(0.6, -0.8);
    bsc.evolve(bham_c, t, 0.0, krydim, tol);
    bsg.evolve(bham_g, t, 0.0, krydim, tol);
    const double block_evolve = std::max(rel_diff(bsg.L, bsc.L), rel_diff(bsg.R, bsc.R));

    std::printf(
        "{\"block_terms\": %.3e, \"otoc_block\": %.3e, \"F_block\": [%.12e, %.12e], "
        "\"block_evolve\": %.3e, ", bterms, otoc_block, (double)Fbc.real(), (double)Fbc.imag(),
        block_evolve);
    std::printf(
        "\"E0_ed_b200\": %.15e, \"ed_overlap\": %.15f, \"ed_evolve\": %.3e, "
        "\"ed_evolve_cached\": %.3e, \"ed_cache_bytes\": %.0f, \"ed_beta\": %.3e, "
        "\"ed_cpu\": %d, \"E0_ed_cpu\": %.15e, \"ed_vs_cpu_ed\": %.3e, ",
        Eed, ed_overlap, ed_evolve, ed_cached, ed_cache_bytes, ed_beta, ed_cpu, ed_cpu_energy,
        ed_cpu_evolve);
    std::printf(
        "\"N\": %d, \"terms\": %zu, \"term_diff\": %.3e, \"roundtrip\": %.3e, \"elem\": %.3e, "
        "\"apply\": %.3e, \"evolve_ref_krylov\": %.3e, \"evolve_b200krylov\": %.3e, "
        "\"evolve_beta\": %.3e, \"otoc\": %.3e, \"F\": [%.12e, %.12e], \"mutate\": %.3e, "
        "\"moved\": %.3e, "
        "\"E0_cpu\": %.15e, \"E0_b200\": %.15e, \"ground_overlap\": %.15f}\n",
        N, ham_c.size(), terms, roundtrip, elem, apply, evolve, evolve_fused, evolve_beta, otoc,
        (double)Fc.real(), (double)Fc.imag(), mutate, moved, Ec, Eg, overlap);
    return 0;
}
