/* rpb200_impl.hpp -- the reference library's backend, rebuilt on librpb200.
 *
 * REAPERS selects its backend at compile time: State<Fp, Impl>,
 * Krylov<Impl> and SYK<Fp, Impl> are templates over an Impl class of static
 * vector operations plus a SumOps type (the concept CPUImpl and GPUImpl
 * implement, inc/cpuimpl.h:509-756 and inc/gpuimpl.h:395-1105).  B200Impl
 * implements that concept on the C ABI of include/rpb200.h, so the
 * reference's own host code runs its hot path on the sm_100a kernels:
 *
 *     #define REAPERS_NOGPU
 *     #include <reapers.h>
 *     #include <rpb200_impl.hpp>
 *     using namespace REAPERS;
 *     State<double, B200Impl> psi(len);
 *     psi.random_state();
 *     psi.evolve(ham, t);                           // the reference's Krylov
 *     psi.evolve<EvolutionAlgorithm::B200Krylov>(ham, t, 0.0, krydim, tol);
 *                                                   // the GPU-resident Krylov
 *
 * Link with -lrpb200.  Vectors live in device memory; element access goes
 * through a proxy that copies one element (as GPUImpl's DeviceVec does).
 * Exact diagonalisation (ExactDiagonalization<B200Impl>, inc/algo.h:29-54)
 * runs on the device as on the reference's GPU backend: B200SumOps builds
 * the dense matrix and its eigensystem (rp_dense_*), matexp results are
 * device matrices kept in the reference's own MatexpCache, and B200Impl's
 * mat_mul and eigenvector copy_vec work on them.
 */
#pragma once

#ifndef _REAPERS_H_
#error "include the reference's reapers.h (with REAPERS_NOGPU) before rpb200_impl.hpp"
#endif

#include <complex>
#include <cstdint>
#include <memory>
#include <random>
#include <tuple>
#include <string>
#include <type_traits>
#include <utility>

#include "rpb200.h"

namespace REAPERS {

namespace b200 {

/* ABI status -> the reference's exception classes (inc/except.h). */
inline void check(int rc, std::size_t bytes = 0) {
    if (rc == RP_OK) return;
    const char *msg = rp_last_error();
    switch (rc) {
    case RP_E_INVALID:
        throw InvalidArgument(__FILE__, __LINE__, __func__, msg);
    case RP_E_NOMEM:
        throw DevOutOfMem(__FILE__, __LINE__, __func__, bytes);
    case RP_E_NODEVICE:
        throw NoGpuDevice(__FILE__, __LINE__, __func__);
    default:
        throw RuntimeError(__FILE__, __LINE__, __func__, "librpb200", rc);
    }
}

template <RealScalar Fp>
constexpr int code() {
    return std::is_same_v<Fp, double> ? RP_C128 : RP_C64;
}

/* Seeds for init_random: fresh per call, like CPUImpl's random_device-seeded
 * generator (inc/cpuimpl.h:539-546). */
inline uint64_t next_seed() {
    static std::mt19937_64 gen{std::random_device{}()};
    return gen();
}

}  // namespace b200

class B200Impl;

/* A state vector in device memory (GPUImpl::DeviceVec, inc/gpuimpl.h:400-494). */
template <RealScalar FpType>
class B200Vec {
    friend class B200Impl;
    std::size_t dim = 0;
    void *p = nullptr;

    B200Vec(const B200Vec &) = delete;
    B200Vec &operator=(const B200Vec &) = delete;

public:
    /* Read or write one element (a one-element copy each way). */
    class ElemRef {
        void *p;
    public:
        explicit ElemRef(void *p) : p(p) {}
        operator complex<FpType>() const {
            complex<FpType> v;
            b200::check(rp_memcpy(&v, p, sizeof(v), 1));
            return v;
        }
        ElemRef &operator=(complex<FpType> v) {
            b200::check(rp_memcpy(p, &v, sizeof(v), 0));
            return *this;
        }
    };

    explicit B200Vec(std::size_t dim) : dim(dim) {
        b200::check(rp_alloc(&p, dim * sizeof(complex<FpType>)), dim * sizeof(complex<FpType>));
    }
    B200Vec(B200Vec &&o) noexcept : dim(o.dim), p(o.p) {
        o.p = nullptr;
        o.dim = 0;
    }
    B200Vec &operator=(B200Vec &&o) noexcept {
        std::swap(dim, o.dim);
        std::swap(p, o.p);
        return *this;
    }
    ~B200Vec() {
        if (p) rp_free(p);
    }
    friend void swap(B200Vec &a, B200Vec &b) noexcept {
        std::swap(a.dim, b.dim);
        std::swap(a.p, b.p);
    }

    /* Conversions with the host backend's vectors, used by State's
     * conversion constructor between backends (inc/state.h:112-118). */
    template <RealScalar FpType1>
    explicit B200Vec(const typename CPUImpl::template VecType<FpType1> &h) : B200Vec(h.dimension()) {
        if constexpr (std::is_same_v<FpType, FpType1>) {
            b200::check(rp_memcpy(p, h.get(), dim * sizeof(complex<FpType>), 0));
        } else {
            B200Vec<FpType1> tmp(h);
            b200::check(rp_vec_copy(b200::code<FpType>(), p, b200::code<FpType1>(), tmp.ptr(), dim));
        }
    }
    template <RealScalar FpType1>
    explicit operator typename CPUImpl::template VecType<FpType1>() const {
        typename CPUImpl::template VecType<FpType1> h(dim);
        if constexpr (std::is_same_v<FpType, FpType1>) {
            b200::check(rp_memcpy(h.get(), p, dim * sizeof(complex<FpType>), 1));
        } else {
            B200Vec<FpType1> tmp(dim);
            b200::check(rp_vec_copy(b200::code<FpType1>(), tmp.ptr(), b200::code<FpType>(), p, dim));
            b200::check(rp_memcpy(h.get(), tmp.ptr(), dim * sizeof(complex<FpType1>), 1));
        }
        return h;
    }

    ElemRef operator[](std::size_t i) { return ElemRef(static_cast<complex<FpType> *>(p) + i); }
    complex<FpType> operator[](std::size_t i) const {
        return ElemRef(static_cast<complex<FpType> *>(p) + i);
    }
    /* State::buf() hands out the vector itself (BufType is a reference). */
    B200Vec &get() { return *this; }
    const B200Vec &get() const { return *this; }
    void *ptr() const { return p; }
    std::size_t dimension() const { return dim; }
};

/* A dense complex matrix in device memory, column-major (the role of
 * DevSumOps::MatrixType, inc/gpuimpl.h:139-300): matexp results and the
 * eigenvector matrix.  A view does not own its memory (the eigenvectors of
 * an rp_dense_t); copies are owning device copies. */
template <RealScalar FpType>
class B200Mat {
    std::size_t rdim = 0, cdim = 0;
    void *p = nullptr;
    bool owns = false;

public:
    B200Mat() = default;
    B200Mat(std::size_t rows, std::size_t cols) : rdim(rows), cdim(cols), owns(true) {
        const std::size_t b = rows * cols * sizeof(complex<FpType>);
        b200::check(rp_alloc(&p, b), b);
    }
    static B200Mat view(void *ptr, std::size_t rows, std::size_t cols) {
        B200Mat m;
        m.rdim = rows;
        m.cdim = cols;
        m.p = ptr;
        return m;
    }
    B200Mat(const B200Mat &o) : B200Mat(o.rdim, o.cdim) {
        if (size()) b200::check(rp_memcpy(p, o.p, size() * sizeof(complex<FpType>), 2));
    }
    B200Mat(B200Mat &&o) noexcept : rdim(o.rdim), cdim(o.cdim), p(o.p), owns(o.owns) {
        o.p = nullptr;
        o.owns = false;
        o.rdim = o.cdim = 0;
    }
    B200Mat &operator=(B200Mat o) noexcept {
        std::swap(rdim, o.rdim);
        std::swap(cdim, o.cdim);
        std::swap(p, o.p);
        std::swap(owns, o.owns);
        return *this;
    }
    ~B200Mat() {
        if (owns && p) rp_free(p);
    }
    std::size_t rows() const { return rdim; }
    std::size_t cols() const { return cdim; }
    /* elements (MatexpCache accounts sizeof(complex) * size() bytes) */
    std::size_t size() const { return rdim * cdim; }
    void *ptr() const { return p; }
};

/* A sum of spin operators whose device table (grouped terms) is built on the
 * first apply and dropped on every change, as DevSumOps does with its device
 * copy (inc/gpuimpl.h:124-395, upload/release at 1065-1105). */
template <RealScalar FpType>
class B200SumOps : public HostSumOps<FpType> {
    friend class B200Impl;
    friend class HostSumOps<FpType>;   // its _matexp_helper reads our cache
    using Impl = B200Impl;

public:
    using MatrixType = B200Mat<FpType>;
    using EigenVals = typename HostSumOps<FpType>::EigenVals;
    using EigenVecs = B200Mat<FpType>;
    using EigenSystem = std::tuple<const EigenVals &, const EigenVecs &>;

private:
    mutable rp_ham_t ham = nullptr;
    mutable int ham_len = -1;
    // exact diagonalisation: the device eigensystem and the matexp results
    mutable rp_dense_t dense = nullptr;
    mutable int dense_len = -1;
    mutable EigenVals dense_evals;
    mutable EigenVecs dense_vecs;
    mutable MatexpCache<FpType, MatrixType, B200Impl> matexp_cache;

    void drop() const {
        if (ham) rp_ham_destroy(ham);
        ham = nullptr;
        ham_len = -1;
        matexp_cache.clear();
        dense_vecs = EigenVecs();
        if (dense) rp_dense_destroy(dense);
        dense = nullptr;
        dense_len = -1;
    }

    /* bit strings and the coefficients the kernels take (sigma_y as sx.sz
     * with its i in the coefficient, inc/ops.h:285-288 and 366-377) */
    void term_arrays(std::vector<uint64_t> &bits, std::vector<double> &coeff) const {
        for (const auto &op : *this) {
            const uint64_t b = (uint64_t)op.get_bit_string();
            const uint64_t xb = b & 0x5555555555555555ull, zb = (b >> 1) & 0x5555555555555555ull;
            const int ny = __builtin_popcountll(xb & zb) & 3;
            std::complex<double> c(op.coefficient().real(), op.coefficient().imag());
            static const std::complex<double> ipow[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
            c *= ipow[ny];
            bits.push_back(b);
            coeff.push_back(c.real());
            coeff.push_back(c.imag());
        }
    }

    /* exp(c H) on the device (DevSumOps::_matexp, inc/gpuimpl.h:1244-1263) */
    MatrixType _matexp(complex<FpType> c, int len) const {
        get_eigensystem(len);
        MatrixType res(dense_vecs.rows(), dense_vecs.cols());
        b200::check(rp_dense_expm(dense, (double)c.real(), (double)c.imag(), res.ptr()));
        return res;
    }

protected:
    void release() const override {
        drop();
        HostSumOps<FpType>::release();
    }
    void mini_release() const override {
        matexp_cache.clear();
        HostSumOps<FpType>::mini_release();
    }

public:
    B200SumOps(const SpinOp<FpType> &op) : HostSumOps<FpType>(op) {}
    B200SumOps(const HostSumOps<FpType> &ops) : HostSumOps<FpType>(ops) {}
    B200SumOps(const B200SumOps &ops) : HostSumOps<FpType>(ops) {}
    /* The reference's HostSumOps moves its term list without a release();
     * the device tables built for a list stay with neither object, so both
     * sides rebuild them on their next use. */
    B200SumOps(B200SumOps &&ops) : HostSumOps<FpType>(std::move(ops)) { ops.drop(); }
    template <RealScalar FpType1>
    explicit B200SumOps(const B200SumOps<FpType1> &ops) : HostSumOps<FpType>(ops) {}
    B200SumOps(const std::initializer_list<SpinOp<FpType>> &l = {}) : HostSumOps<FpType>(l) {}
    using HostSumOps<FpType>::operator=;
    B200SumOps &operator=(const B200SumOps &rhs) {
        HostSumOps<FpType>::operator=(rhs);
        return *this;
    }
    B200SumOps &operator=(B200SumOps &&rhs) {
        if (this != &rhs) {
            drop();
            rhs.drop();
            HostSumOps<FpType>::operator=(static_cast<HostSumOps<FpType> &&>(rhs));
        }
        return *this;
    }
    ~B200SumOps() { drop(); }

    /* The library's grouped term table for a chain of len sites. */
    rp_ham_t handle(int len) const {
        if (ham && ham_len == len) return ham;
        if (ham) rp_ham_destroy(ham);
        ham = nullptr;
        ham_len = -1;
        std::vector<uint64_t> bits;
        std::vector<double> coeff;
        term_arrays(bits, coeff);
        rp_ham_t h = nullptr;
        b200::check(rp_ham_create(&h, len, b200::code<FpType>(), bits.size(), bits.data(),
                                  coeff.data()));
        ham = h;
        ham_len = len;
        return ham;
    }

    /* The eigensystem of the (Hermitian) operator on len sites, computed on
     * the device once per len (DevSumOps::get_eigensystem,
     * inc/gpuimpl.h:1180-1240): eigenvalues ascending on the host, the
     * eigenvectors the columns of a device matrix. */
    EigenSystem get_eigensystem(int len) const {
        if (!dense || dense_len != len) {
            matexp_cache.clear();
            dense_vecs = EigenVecs();
            if (dense) rp_dense_destroy(dense);
            dense = nullptr;
            dense_len = -1;
            std::vector<uint64_t> bits;
            std::vector<double> coeff;
            term_arrays(bits, coeff);
            rp_dense_t d = nullptr;
            b200::check(rp_dense_create(&d, len, b200::code<FpType>(), bits.size(), bits.data(),
                                        coeff.data()));
            dense = d;
            dense_len = len;
            const std::size_t dim = std::size_t(1) << len;
            std::vector<double> ev(dim);
            b200::check(rp_dense_eigenvalues(dense, ev.data()));
            dense_evals.resize(dim, 1);
            for (std::size_t i = 0; i < dim; i++) dense_evals(i, 0) = (FpType)ev[i];
            void *vp = nullptr;
            b200::check(rp_dense_eigenvectors(dense, &vp));
            dense_vecs = EigenVecs::view(vp, dim, dim);
        }
        return {dense_evals, dense_vecs};
    }

    /* exp(c H) for a chain of len sites, kept in the reference's MatexpCache
     * (inc/cpuimpl.h:25-88) by its HostSumOps::_matexp_helper. */
    const MatrixType &matexp(complex<FpType> c, int len) const {
        return HostSumOps<FpType>::_matexp_helper(*this, c, len);
    }
};

/* The backend: the statics State, Krylov and SYK call (inc/cpuimpl.h:582-754). */
class B200Impl {
public:
    template <RealScalar FpType>
    using VecType = B200Vec<FpType>;
    template <RealScalar FpType>
    using VecSizeType = typename SpinOp<FpType>::StateType;
    template <RealScalar FpType>
    using BufType = B200Vec<FpType> &;
    template <RealScalar FpType>
    using ConstBufType = const B200Vec<FpType> &;
    template <RealScalar FpType>
    using ElemRefType = typename B200Vec<FpType>::ElemRef;
    template <RealScalar FpType>
    using SumOps = B200SumOps<FpType>;

    /* Haar-random state: Gaussian entries, normalised (inc/cpuimpl.h:601-611). */
    template <RealScalar FpType>
    static void init_random(VecSizeType<FpType> size, BufType<FpType> v) {
        b200::check(rp_vec_random(b200::code<FpType>(), size, v.ptr(), b200::next_seed()));
        double n = 0;
        b200::check(rp_vec_norm(b200::code<FpType>(), size, v.ptr(), &n));
        b200::check(rp_vec_scale(b200::code<FpType>(), size, v.ptr(), 1.0 / n, 0.0));
    }

    template <RealScalar FpType>
    static void zero_vec(VecSizeType<FpType> size, BufType<FpType> v) {
        b200::check(rp_vec_zero(b200::code<FpType>(), size, v.ptr()));
    }

    template <RealScalar FpType0, RealScalar FpType1>
    static void copy_vec(VecSizeType<FpType0> size, BufType<FpType0> v0, ConstBufType<FpType1> v1) {
        b200::check(rp_vec_copy(b200::code<FpType0>(), v0.ptr(), b200::code<FpType1>(), v1.ptr(), size));
    }

    /* v0 += v1 */
    template <RealScalar FpType>
    static void add_vec(VecSizeType<FpType> size, BufType<FpType> v0, ConstBufType<FpType> v1) {
        b200::check(rp_vec_axpy(b200::code<FpType>(), size, v0.ptr(), 1.0, 0.0, v1.ptr()));
    }
    /* v0 += s * v1 */
    template <RealScalar FpType>
    static void add_vec(VecSizeType<FpType> size, BufType<FpType> v0, FpType s, ConstBufType<FpType> v1) {
        b200::check(rp_vec_axpy(b200::code<FpType>(), size, v0.ptr(), s, 0.0, v1.ptr()));
    }
    template <RealScalar FpType>
    static void add_vec(VecSizeType<FpType> size, BufType<FpType> v0, complex<FpType> s,
                        ConstBufType<FpType> v1) {
        b200::check(rp_vec_axpy(b200::code<FpType>(), size, v0.ptr(), s.real(), s.imag(), v1.ptr()));
    }
    /* res = v0 + v1 */
    template <RealScalar FpType>
    static void add_vec(VecSizeType<FpType> size, BufType<FpType> res, ConstBufType<FpType> v0,
                        ConstBufType<FpType> v1) {
        b200::check(rp_vec_add(b200::code<FpType>(), size, res.ptr(), v0.ptr(), v1.ptr()));
    }

    template <RealScalar FpType>
    static void scale_vec(VecSizeType<FpType> size, BufType<FpType> v, FpType s) {
        b200::check(rp_vec_scale(b200::code<FpType>(), size, v.ptr(), s, 0.0));
    }
    template <RealScalar FpType>
    static void scale_vec(VecSizeType<FpType> size, BufType<FpType> v, complex<FpType> s) {
        b200::check(rp_vec_scale(b200::code<FpType>(), size, v.ptr(), s.real(), s.imag()));
    }

    /* <v0|v1>, FP64 with compensated summation on the GPU */
    template <RealScalar FpType>
    static complex<FpType> vec_prod(VecSizeType<FpType> size, ConstBufType<FpType> v0,
                                    ConstBufType<FpType> v1) {
        double r[2];
        b200::check(rp_vec_dot(b200::code<FpType>(), size, v0.ptr(), v1.ptr(), r));
        return complex<FpType>{FpType(r[0]), FpType(r[1])};
    }

    template <RealScalar FpType>
    static FpType vec_norm(VecSizeType<FpType> size, ConstBufType<FpType> v) {
        double n = 0;
        b200::check(rp_vec_norm(b200::code<FpType>(), size, v.ptr(), &n));
        return FpType(n);
    }

    /* res = mat * vec for a device matrix (GPUImpl::mat_mul,
     * inc/gpuimpl.h:1012-1021; ExactDiagonalization::evolve) */
    template <RealScalar FpType>
    static void mat_mul(VecSizeType<FpType> dim, BufType<FpType> res, const B200Mat<FpType> &mat,
                        ConstBufType<FpType> vec) {
        if (mat.rows() != dim || mat.cols() != dim)
            throw InvalidArgument(__FILE__, __LINE__, __func__, "matrix and vector sizes differ");
        b200::check(rp_mat_vec(b200::code<FpType>(), dim, mat.ptr(), vec.ptr(), res.ptr()));
    }

    /* res = column col of a device matrix (the eigenvector copy of
     * ExactDiagonalization::ground_state; GPUImpl::copy_vec,
     * inc/gpuimpl.h:894-900) */
    template <RealScalar FpType>
    static void copy_vec(VecSizeType<FpType> size, BufType<FpType> res, const B200Mat<FpType> &mat,
                         ssize_t col) {
        if (col < 0 || (std::size_t)col >= mat.cols() || mat.rows() != size)
            throw InvalidArgument(__FILE__, __LINE__, __func__, "eigenvector index out of range");
        const std::size_t b = size * sizeof(complex<FpType>);
        b200::check(rp_memcpy(res.ptr(), static_cast<char *>(mat.ptr()) + (std::size_t)col * b, b, 2));
    }

    /* Device memory budget of the matexp cache (the reference's
     * cache_reserve / cache_release / set_max_cache_size, inc/gpuimpl.h:560-590). */
    inline static std::size_t max_cache_size = std::size_t(16) << 30;
    inline static std::size_t cache_size = 0;
    static bool cache_reserve(std::size_t sz) {
        if (cache_size + sz > max_cache_size) return false;
        cache_size += sz;
        return true;
    }
    static void cache_release(std::size_t sz) { cache_size -= sz <= cache_size ? sz : cache_size; }
    static void set_max_cache_size(std::size_t sz) { max_cache_size = sz; }
    static std::size_t get_max_cache_size() { return max_cache_size; }
    static std::size_t get_current_cache_size() { return cache_size; }
    static int get_device_count() {
        int n = 0;
        b200::check(rp_device_count(&n));
        return n;
    }

    /* res += ops * vec (inc/cpuimpl.h:738-754, src/krnl.cu:220-257) */
    template <RealScalar FpType>
    static void apply_ops(typename SpinOp<FpType>::IndexType len, BufType<FpType> res,
                          const B200SumOps<FpType> &ops, ConstBufType<FpType> vec) {
        b200::check(rp_apply(ops.handle(len), res.ptr(), vec.ptr(), 1));
    }
};

namespace EvolutionAlgorithm {

/* The restarted Krylov of Krylov<Impl>::evolve (inc/algo.h:267-365) as one
 * library call: the Arnoldi cycles, Hfull and its exponential stay on the
 * GPU.  Selected with State::evolve<B200Krylov>(ham, t, beta, krydim, tol,
 * max_iters); the arguments and defaults are Krylov's. */
template <typename Impl>
struct B200Krylov {
    static_assert(std::is_same_v<Impl, B200Impl>, "B200Krylov runs on B200Impl states");

    template <RealScalar FpType>
    static void evolve(State<FpType, Impl> &s, const B200SumOps<FpType> &ops, FpType t,
                       FpType beta, int krydim = 5, FpType tol = epsilon<FpType>(),
                       int max_iters = 0) {
        rp_evolve_stats_t st;
        b200::check(rp_evolve(ops.handle(s.spin_chain_length()), s.buf().ptr(), (double)t,
                              (double)beta, krydim, (double)tol, max_iters, &st));
    }
};

}  // namespace EvolutionAlgorithm

}  // namespace REAPERS
