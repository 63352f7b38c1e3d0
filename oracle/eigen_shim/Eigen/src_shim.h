// Minimal Eigen-API subset, written for this project so that the REAPERS
// headers (which include <Eigen/Eigen>, <Eigen/Eigenvalues> and
// <unsupported/Eigen/MatrixFunctions> unconditionally) can be compiled as a
// CPU oracle on a machine without Eigen3.  TEST INFRASTRUCTURE ONLY.
//
// Only what the REAPERS CPU path instantiates is provided: dynamic
// column-major matrices and vectors, Map, products, adjoint, asDiagonal,
// unaryExpr, minCoeff, conservativeResize, comma initialisation, a
// Hermitian eigen-solver (cyclic Jacobi) and the matrix exponential.
//
// The matrix exponential follows the published method N. J. Higham, "The
// scaling and squaring method for the matrix exponential revisited", SIAM J.
// Matrix Anal. Appl. 26(4):1179-1193, 2005: Pade degree 3/5/7/9/13 selected by
// the 1-norm thresholds theta_m, scaling and squaring for degree 13.  Results
// agree with other implementations of that method to rounding, not bitwise.
#pragma once

// Eigen pulls these standard headers in transitively and the REAPERS headers
// rely on that.

#include <algorithm>
#include <cassert>
#include <cmath>
#include <complex>
#include <cstddef>
#include <initializer_list>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace Eigen {

constexpr int Dynamic = -1;
enum ComputationInfo { Success = 0, NumericalIssue = 1, NoConvergence = 2 };
enum DecompositionOptions { ComputeEigenvectors = 1, EigenvaluesOnly = 2 };
using Index = std::ptrdiff_t;

namespace shim {
template <typename T> struct real_of { using type = T; };
template <typename T> struct real_of<std::complex<T>> { using type = T; };
template <typename T> inline T conj_of(const T &v) { return v; }
template <typename T> inline std::complex<T> conj_of(const std::complex<T> &v) { return std::conj(v); }
template <typename T> inline typename real_of<T>::type abs2(const T &v) { return std::norm(std::complex<typename real_of<T>::type>(v)); }
}  // namespace shim

template <typename T, int Rows = Dynamic, int Cols = Dynamic>
class Matrix;

// Comma initialiser: m << a, b, c;  fills row by row.
template <typename M>
class CommaInit {
    M &m;
    Index k;
public:
    CommaInit(M &m, const typename M::Scalar &v) : m(m), k(0) { put(v); }
    void put(const typename M::Scalar &v) {
        Index r = k / m.cols(), c = k % m.cols();
        m(r, c) = v;
        k++;
    }
    CommaInit &operator,(const typename M::Scalar &v) { put(v); return *this; }
};

template <typename T, int Rows, int Cols>
class Matrix {
    Index nr = 0, nc = 0;
    std::vector<T> d;
public:
    using Scalar = T;
    using RealScalar = typename shim::real_of<T>::type;

    Matrix() : nr(Rows == Dynamic ? 0 : Rows), nc(Cols == Dynamic ? 0 : Cols),
               d((size_t)nr * nc) {}
    Matrix(Index r, Index c) : nr(r), nc(c), d((size_t)r * c) {}
    template <int R = Rows, int C = Cols, typename = std::enable_if_t<(C == 1 || R == 1)>>
    explicit Matrix(Index n) : nr(Cols == 1 ? n : 1), nc(Cols == 1 ? 1 : n), d((size_t)n) {}
    template <typename Other, typename = decltype(std::declval<const Other &>().rows()),
              typename = std::enable_if_t<!std::is_same_v<std::decay_t<Other>, Matrix>>>
    Matrix(const Other &o) : nr(o.rows()), nc(o.cols()), d((size_t)o.rows() * o.cols()) {
        for (Index j = 0; j < nc; j++)
            for (Index i = 0; i < nr; i++) (*this)(i, j) = o(i, j);
    }
    Matrix(const Matrix &) = default;
    Matrix(Matrix &&) = default;
    Matrix &operator=(const Matrix &) = default;
    Matrix &operator=(Matrix &&) = default;
    template <typename Other, typename = decltype(std::declval<const Other &>().rows()),
              typename = std::enable_if_t<!std::is_same_v<std::decay_t<Other>, Matrix>>>
    Matrix &operator=(const Other &o) {
        Matrix tmp(o);
        *this = std::move(tmp);
        return *this;
    }

    Index rows() const { return nr; }
    Index cols() const { return nc; }
    Index size() const { return nr * nc; }
    T *data() { return d.data(); }
    const T *data() const { return d.data(); }
    T &operator()(Index i, Index j) { return d[(size_t)j * nr + i]; }
    const T &operator()(Index i, Index j) const { return d[(size_t)j * nr + i]; }
    T &operator()(Index i) { return d[(size_t)i]; }
    const T &operator()(Index i) const { return d[(size_t)i]; }
    T &operator[](Index i) { return d[(size_t)i]; }
    const T &operator[](Index i) const { return d[(size_t)i]; }

    void resize(Index r, Index c) {
        if (r * c != nr * nc) d.assign((size_t)r * c, T{});
        nr = r;
        nc = c;
    }
    void resize(Index n) { resize(Cols == 1 ? n : 1, Cols == 1 ? 1 : n); }
    void conservativeResize(Index r, Index c) {
        std::vector<T> nd((size_t)r * c, T{});
        for (Index j = 0; j < std::min(c, nc); j++)
            for (Index i = 0; i < std::min(r, nr); i++) nd[(size_t)j * r + i] = (*this)(i, j);
        d.swap(nd);
        nr = r;
        nc = c;
    }
    Matrix &setZero() { std::fill(d.begin(), d.end(), T{}); return *this; }
    static Matrix Zero(Index r, Index c) { return Matrix(r, c); }
    static Matrix Identity(Index r, Index c) {
        Matrix m(r, c);
        for (Index i = 0; i < std::min(r, c); i++) m(i, i) = T(1);
        return m;
    }
    CommaInit<Matrix> operator<<(const T &v) { return CommaInit<Matrix>(*this, v); }

    Matrix<T, Dynamic, 1> col(Index j) const {
        Matrix<T, Dynamic, 1> v(nr, 1);
        for (Index i = 0; i < nr; i++) v(i, 0) = (*this)(i, j);
        return v;
    }
    RealScalar squaredNorm() const {
        RealScalar s = 0;
        for (auto &v : d) s += shim::abs2(v);
        return s;
    }
    RealScalar norm() const { return std::sqrt(squaredNorm()); }
    Matrix adjoint() const {
        Matrix a(nc, nr);
        for (Index j = 0; j < nc; j++)
            for (Index i = 0; i < nr; i++) a(j, i) = shim::conj_of((*this)(i, j));
        return a;
    }
    Matrix transpose() const {
        Matrix a(nc, nr);
        for (Index j = 0; j < nc; j++)
            for (Index i = 0; i < nr; i++) a(j, i) = (*this)(i, j);
        return a;
    }
    T trace() const {
        T s{};
        for (Index i = 0; i < std::min(nr, nc); i++) s += (*this)(i, i);
        return s;
    }
    template <typename F>
    auto unaryExpr(F f) const {
        using R = std::decay_t<decltype(f(std::declval<T>()))>;
        Matrix<R, Rows, Cols> out(nr, nc);
        for (Index j = 0; j < nc; j++)
            for (Index i = 0; i < nr; i++) out(i, j) = f((*this)(i, j));
        return out;
    }
    T minCoeff(Index *r, Index *c) const {
        Index br = 0, bc = 0;
        for (Index j = 0; j < nc; j++)
            for (Index i = 0; i < nr; i++)
                if ((*this)(i, j) < (*this)(br, bc)) { br = i; bc = j; }
        *r = br;
        *c = bc;
        return (*this)(br, bc);
    }
    template <typename I>
    T minCoeff(I *idx) const {
        Index best = 0;
        for (Index i = 1; i < size(); i++)
            if (d[(size_t)i] < d[(size_t)best]) best = i;
        *idx = (I)best;
        return d[(size_t)best];
    }
    Matrix &operator+=(const Matrix &o) { for (size_t i = 0; i < d.size(); i++) d[i] += o.d[i]; return *this; }
    Matrix &operator-=(const Matrix &o) { for (size_t i = 0; i < d.size(); i++) d[i] -= o.d[i]; return *this; }
    Matrix operator-(const Matrix &o) const { Matrix r(*this); r -= o; return r; }
    Matrix operator+(const Matrix &o) const { Matrix r(*this); r += o; return r; }
    Matrix operator-() const { Matrix r(*this); for (auto &v : r.d) v = -v; return r; }
    bool operator==(const Matrix &o) const { return nr == o.nr && nc == o.nc && d == o.d; }
    bool operator!=(const Matrix &o) const { return !(*this == o); }

    // Diagonal wrapper for vectors.
    struct Diag {
        const Matrix &v;
        Index rows() const { return v.size(); }
        Index cols() const { return v.size(); }
        T operator()(Index i, Index j) const { return i == j ? v[i] : T{}; }
    };
    Diag asDiagonal() const { return Diag{*this}; }

    // Matrix exponential (Higham 2005).
    Matrix exp() const;
};

template <typename M>
class Map {
    using T = typename M::Scalar;
    using PT = std::conditional_t<std::is_const_v<M>, const T *, T *>;
    PT p;
    Index nr, nc;
public:
    using Scalar = std::remove_const_t<T>;
    Map(PT p, Index r, Index c) : p(p), nr(r), nc(c) {}
    Map(PT p, Index n) : p(p), nr(n), nc(1) {}
    Index rows() const { return nr; }
    Index cols() const { return nc; }
    Index size() const { return nr * nc; }
    const T &operator()(Index i, Index j) const { return p[(size_t)j * nr + i]; }
    template <typename Q = M, typename = std::enable_if_t<!std::is_const_v<Q>>>
    T &operator()(Index i, Index j) { return p[(size_t)j * nr + i]; }
    const T &operator[](Index i) const { return p[(size_t)i]; }
    template <typename Other>
    Map &operator=(const Other &o) {
        // evaluate first (the right-hand side may alias the destination)
        std::remove_const_t<M> tmp(o);
        for (Index j = 0; j < nc; j++)
            for (Index i = 0; i < nr; i++) p[(size_t)j * nr + i] = tmp(i, j);
        return *this;
    }
};

// Generic product of two matrix-like objects; the inner loop runs down
// columns of the left operand (column-major friendly).
template <typename A, typename B,
          typename = decltype(std::declval<const A &>().rows()),
          typename = decltype(std::declval<const B &>().cols())>
auto operator*(const A &a, const B &b) {
    using TA = std::decay_t<decltype(a(0, 0))>;
    using TB = std::decay_t<decltype(b(0, 0))>;
    using T = decltype(std::declval<TA>() * std::declval<TB>());
    Matrix<T, Dynamic, Dynamic> c(a.rows(), b.cols());
    Index n = a.rows(), kk = a.cols(), m = b.cols();
    if (m == 1 && n >= 1024) {
        #pragma omp parallel for schedule(static)
        for (Index i = 0; i < n; i++) {
            T s{};
            for (Index k = 0; k < kk; k++) s += a(i, k) * b(k, 0);
            c(i, 0) = s;
        }
        return c;
    }
    for (Index j = 0; j < m; j++)
        for (Index k = 0; k < kk; k++) {
            T bk = b(k, j);
            for (Index i = 0; i < n; i++) c(i, j) += a(i, k) * bk;
        }
    return c;
}

template <typename S, typename T, int R, int C,
          typename = std::enable_if_t<std::is_convertible_v<S, T>>>
Matrix<T, R, C> operator*(const S &s, const Matrix<T, R, C> &m) {
    Matrix<T, R, C> r(m);
    for (Index j = 0; j < r.cols(); j++)
        for (Index i = 0; i < r.rows(); i++) r(i, j) = T(s) * r(i, j);
    return r;
}

namespace shim {
template <typename T>
using CM = Matrix<T, Dynamic, Dynamic>;

template <typename T>
typename real_of<T>::type norm1(const CM<T> &a) {
    typename real_of<T>::type best = 0;
    for (Index j = 0; j < a.cols(); j++) {
        typename real_of<T>::type s = 0;
        for (Index i = 0; i < a.rows(); i++) s += std::abs(a(i, j));
        best = std::max(best, s);
    }
    return best;
}

// Solve Q X = P (Gaussian elimination, partial pivoting); returns X.
template <typename T>
CM<T> solve(CM<T> Q, CM<T> P) {
    Index n = Q.rows();
    for (Index k = 0; k < n; k++) {
        Index p = k;
        auto best = std::abs(Q(k, k));
        for (Index i = k + 1; i < n; i++)
            if (std::abs(Q(i, k)) > best) { best = std::abs(Q(i, k)); p = i; }
        if (p != k) {
            for (Index j = 0; j < n; j++) std::swap(Q(k, j), Q(p, j));
            for (Index j = 0; j < P.cols(); j++) std::swap(P(k, j), P(p, j));
        }
        T dk = Q(k, k);
        for (Index i = k + 1; i < n; i++) {
            T f = Q(i, k) / dk;
            if (f == T{}) continue;
            for (Index j = k; j < n; j++) Q(i, j) -= f * Q(k, j);
            for (Index j = 0; j < P.cols(); j++) P(i, j) -= f * P(k, j);
        }
    }
    for (Index j = 0; j < P.cols(); j++)
        for (Index i = n - 1; i >= 0; i--) {
            T s = P(i, j);
            for (Index k = i + 1; k < n; k++) s -= Q(i, k) * P(k, j);
            P(i, j) = s / Q(i, i);
        }
    return P;
}
}  // namespace shim

template <typename T, int Rows, int Cols>
Matrix<T, Rows, Cols> Matrix<T, Rows, Cols>::exp() const {
    using R = typename shim::real_of<T>::type;
    using M = shim::CM<T>;
    // Pade numerator coefficients, Higham (2005) Table 2.2 / eq. (2.11).
    static const double b13[14] = {
        64764752532480000.0, 32382376266240000.0, 7771770303897600.0,
        1187353796428800.0, 129060195264000.0, 10559470521600.0, 670442572800.0,
        33522128640.0, 1323241920.0, 40840800.0, 960960.0, 16380.0, 182.0, 1.0};
    static const double b9[10] = {17643225600.0, 8821612800.0, 2075673600.0,
        302702400.0, 30270240.0, 2162160.0, 110880.0, 3960.0, 90.0, 1.0};
    static const double b7[8] = {17297280.0, 8648640.0, 1995840.0, 277200.0,
        25200.0, 1512.0, 56.0, 1.0};
    static const double b5[6] = {30240.0, 15120.0, 3360.0, 420.0, 30.0, 1.0};
    static const double b3[4] = {120.0, 60.0, 12.0, 1.0};
    const double theta[5] = {1.495585217958292e-2, 2.539398330063230e-1,
                             9.504178996162932e-1, 2.097847961257068e0,
                             5.371920351148152e0};
    Index n = nr;
    M A(*this);
    R a1 = shim::norm1(A);
    int s = 0, deg;
    if (a1 <= theta[0]) deg = 3;
    else if (a1 <= theta[1]) deg = 5;
    else if (a1 <= theta[2]) deg = 7;
    else if (a1 <= theta[3]) deg = 9;
    else {
        deg = 13;
        double r = (double)a1 / theta[4];
        if (r > 1) s = (int)std::ceil(std::log2(r));
        R sc = (R)std::ldexp(1.0, -s);
        for (Index j = 0; j < n; j++)
            for (Index i = 0; i < n; i++) A(i, j) = A(i, j) * sc;
    }
    M I = M::Identity(n, n);
    M A2 = A * A;
    M U(n, n), V(n, n);
    if (deg == 13) {
        M A4 = A2 * A2, A6 = A4 * A2;
        M t1 = (R)b13[13] * A6 + (R)b13[11] * A4 + (R)b13[9] * A2;
        M u = A6 * t1 + (R)b13[7] * A6 + (R)b13[5] * A4 + (R)b13[3] * A2 + (R)b13[1] * I;
        U = A * u;
        M t2 = (R)b13[12] * A6 + (R)b13[10] * A4 + (R)b13[8] * A2;
        V = A6 * t2 + (R)b13[6] * A6 + (R)b13[4] * A4 + (R)b13[2] * A2 + (R)b13[0] * I;
    } else {
        const double *b = deg == 3 ? b3 : deg == 5 ? b5 : deg == 7 ? b7 : b9;
        M P = I, odd(n, n);
        for (int k = 0; 2 * k <= deg; k++) {
            V += (R)b[2 * k] * P;
            odd += (R)b[2 * k + 1] * P;
            if (2 * k + 2 <= deg) P = P * A2;
        }
        U = A * odd;
    }
    M E = shim::solve<T>(V - U, V + U);
    for (int k = 0; k < s; k++) E = E * E;
    return Matrix(E);
}

// Hermitian eigen-solver by cyclic Jacobi rotations; eigenvalues ascending.
template <typename MatT>
class SelfAdjointEigenSolver {
public:
    using Scalar = typename MatT::Scalar;
    using R = typename shim::real_of<Scalar>::type;
    using RealVectorType = Matrix<R, Dynamic, 1>;
    using EigenvectorsType = Matrix<Scalar, Dynamic, Dynamic>;
private:
    RealVectorType vals;
    EigenvectorsType vecs;
    ComputationInfo st = Success;

    void run(EigenvectorsType A) {
        Index n = A.rows();
        EigenvectorsType Q = EigenvectorsType::Identity(n, n);
        for (int sweep = 0; sweep < 100; sweep++) {
            R off = 0, tot = 0;
            for (Index j = 0; j < n; j++)
                for (Index i = 0; i < n; i++) {
                    R v = std::abs(A(i, j));
                    tot += v * v;
                    if (i != j) off += v * v;
                }
            if (off <= tot * std::numeric_limits<R>::epsilon() * std::numeric_limits<R>::epsilon()) break;
            for (Index p = 0; p < n; p++)
                for (Index q = p + 1; q < n; q++) {
                    Scalar apq = A(p, q);
                    R mag = std::abs(apq);
                    if (mag == 0) continue;
                    Scalar ph = apq / mag;   // phase of a_pq
                    R app = std::real(A(p, p)), aqq = std::real(A(q, q));
                    R tau = (aqq - app) / (2 * mag);
                    R t = (tau >= 0 ? 1 : -1) / (std::abs(tau) + std::sqrt(1 + tau * tau));
                    R c = 1 / std::sqrt(1 + t * t), sn = t * c;
                    // rotation J = [[c, s*ph], [-s*conj(ph), c]] acting on columns p,q
                    for (Index k = 0; k < n; k++) {
                        Scalar akp = A(k, p), akq = A(k, q);
                        A(k, p) = c * akp - sn * shim::conj_of(ph) * akq;
                        A(k, q) = sn * ph * akp + c * akq;
                    }
                    for (Index k = 0; k < n; k++) {
                        Scalar apk = A(p, k), aqk = A(q, k);
                        A(p, k) = c * apk - sn * ph * aqk;
                        A(q, k) = sn * shim::conj_of(ph) * apk + c * aqk;
                    }
                    for (Index k = 0; k < n; k++) {
                        Scalar qkp = Q(k, p), qkq = Q(k, q);
                        Q(k, p) = c * qkp - sn * shim::conj_of(ph) * qkq;
                        Q(k, q) = sn * ph * qkp + c * qkq;
                    }
                }
        }
        std::vector<Index> order(n);
        for (Index i = 0; i < n; i++) order[i] = i;
        std::sort(order.begin(), order.end(),
                  [&](Index a, Index b) { return std::real(A(a, a)) < std::real(A(b, b)); });
        vals = RealVectorType(n, 1);
        vecs = EigenvectorsType(n, n);
        for (Index i = 0; i < n; i++) {
            vals(i, 0) = std::real(A(order[i], order[i]));
            for (Index k = 0; k < n; k++) vecs(k, i) = Q(k, order[i]);
        }
    }
public:
    SelfAdjointEigenSolver() = default;
    template <typename M>
    explicit SelfAdjointEigenSolver(const M &m, int = ComputeEigenvectors) { run(EigenvectorsType(m)); }
    template <typename VA, typename VB>
    SelfAdjointEigenSolver &computeFromTridiagonal(const VA &diag, const VB &sub, int = ComputeEigenvectors) {
        Index n = diag.size();
        EigenvectorsType A(n, n);
        for (Index i = 0; i < n; i++) A(i, i) = diag(i, 0);
        for (Index i = 0; i + 1 < n; i++) { A(i + 1, i) = sub(i, 0); A(i, i + 1) = sub(i, 0); }
        run(A);
        return *this;
    }
    ComputationInfo info() const { return st; }
    const RealVectorType &eigenvalues() const { return vals; }
    const EigenvectorsType &eigenvectors() const { return vecs; }
};

}  // namespace Eigen
