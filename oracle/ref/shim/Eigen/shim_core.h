// Eigen-API shim used only to compile the reference's own sources into the
// CPU oracle library oracle/_ref/libprism_ref.so (test infrastructure; no
// product code includes it).
//
// The reference (src/prism/types.h:3-4) needs Eigen3, which is absent from this
// image. This header provides the subset of Eigen's documented public API that
// the reference calls -- fixed 3-vectors and 3x3 matrices, dynamic vectors, a
// column-major SparseMatrix<double> with setFromTriplets, and
// BiCGSTAB<SparseMatrix, IncompleteLUT> -- written from Eigen's public
// documentation, evaluated eagerly (no expression templates). Semantics kept
// where they decide results:
//   * SparseMatrix::setFromTriplets sums duplicate entries in insertion order;
//     setZero() removes every stored entry (the pattern is rebuilt by the next
//     sum), A += B stores the union pattern (a + b where both exist);
//   * sparse * dense accumulates each row over increasing column index;
//   * dot products and sums run in index order; 3x3 inverse by cofactors;
//   * BiCGSTAB: van der Vorst (1992), right preconditioned, restart when
//     |r0.r| collapses, default tolerance = machine epsilon, default maximum
//     2n iterations; IncompleteLUT: Saad's ILUT (1994) with Eigen's documented
//     defaults (drop tolerance 1e-12 relative to the row norm, fill factor 10),
//     in the natural ordering (Eigen permutes by AMD first, which changes only
//     the preconditioner, not the converged solution).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <ostream>
#include <stdexcept>
#include <type_traits>
#include <utility>
#include <vector>

namespace Eigen {

using Index = std::ptrdiff_t;
inline constexpr int Dynamic = -1;
inline constexpr int Infinity = -1;
enum StorageOptions { ColMajor = 0, RowMajor = 1 };
enum ComputationInfo { Success = 0, NumericalIssue = 1, NoConvergence = 2, InvalidInput = 3 };

template <typename T>
struct NumTraits {
    static constexpr T epsilon() { return std::numeric_limits<T>::epsilon(); }
    static constexpr T dummy_precision() { return T(1e-12); }
};

template <typename S, int R, int C>
class Matrix;
template <typename S, int R, int C>
class ArrayView;

namespace shim {
template <typename T>
inline constexpr bool is_scalar_v = std::is_arithmetic_v<std::decay_t<T>>;

// Comma initializer writing consecutive coefficients through a setter.
template <typename Target>
class CommaInit {
  public:
    CommaInit(Target& t, Index start) : t_(t), i_(start) {}
    template <typename T>
    CommaInit& operator,(T v) {
        t_.setLinear(i_++, static_cast<double>(v));
        return *this;
    }

  private:
    Target& t_;
    Index i_;
};
} // namespace shim

// Dense matrix / vector, column-major, eager.
template <typename S, int R, int C>
class Matrix {
  public:
    static constexpr bool kFixed = (R != Dynamic && C != Dynamic);
    static constexpr int RowsAtCompileTime = R;
    static constexpr int ColsAtCompileTime = C;
    using Scalar = S;

    Matrix() : r_(R == Dynamic ? 0 : R), c_(C == Dynamic ? 0 : C) { alloc(); }

    // size constructor of dynamic vectors (VectorXd v(n))
    template <typename I, typename = std::enable_if_t<std::is_integral_v<I> && !kFixed>>
    explicit Matrix(I n) {
        if constexpr (C == 1) {
            r_ = static_cast<Index>(n);
            c_ = 1;
        } else if constexpr (R == 1) {
            r_ = 1;
            c_ = static_cast<Index>(n);
        } else {
            r_ = static_cast<Index>(n);
            c_ = (C == Dynamic ? 0 : C);
        }
        alloc();
    }

    // rows x cols constructor of dynamic matrices
    template <typename I, typename J,
              typename = std::enable_if_t<std::is_integral_v<I> && std::is_integral_v<J> && !kFixed &&
                                          R == Dynamic && C != 1>>
    Matrix(I r, J c) : r_(r), c_(c) {
        alloc();
    }

    // coefficient constructor of fixed 3-vectors (Vector3d {x, y, z})
    template <typename A, typename B, typename D,
              typename = std::enable_if_t<kFixed && R * C == 3 && shim::is_scalar_v<A> &&
                                          shim::is_scalar_v<B> && shim::is_scalar_v<D>>>
    Matrix(A x, B y, D z) : r_(R), c_(C) {
        d_[0] = static_cast<S>(x);
        d_[1] = static_cast<S>(y);
        d_[2] = static_cast<S>(z);
    }

    Matrix(const Matrix&) = default;
    Matrix(Matrix&&) noexcept = default;
    Matrix& operator=(const Matrix&) = default;
    Matrix& operator=(Matrix&&) noexcept = default;

    // from an array view (vol.array() / (d.array() + eps))
    Matrix(const ArrayView<S, R, C>& a);  // NOLINT(google-explicit-constructor)

    // dimensions
    Index rows() const { return r_; }
    Index cols() const { return c_; }
    Index size() const { return r_ * c_; }
    void resize(Index n) {
        if constexpr (C == 1) {
            r_ = n;
        } else if constexpr (R == 1) {
            c_ = n;
        } else {
            r_ = n;
        }
        alloc();
    }
    void resize(Index r, Index c) {
        r_ = r;
        c_ = c;
        alloc();
    }
    void conservativeResize(Index n) {
        Matrix old = *this;
        resize(n);
        for (Index i = 0; i < std::min(n, old.size()); ++i) d_[i] = old.d_[i];
    }

    // coefficient access
    S& operator()(Index i) { return d_[i]; }
    const S& operator()(Index i) const { return d_[i]; }
    S& operator()(Index i, Index j) { return d_[i + j * r_]; }
    const S& operator()(Index i, Index j) const { return d_[i + j * r_]; }
    S& operator[](Index i) { return d_[i]; }
    const S& operator[](Index i) const { return d_[i]; }
    S& coeffRef(Index i) { return d_[i]; }
    S coeff(Index i) const { return d_[i]; }
    S coeff(Index i, Index j) const { return d_[i + j * r_]; }
    S& x() { return d_[0]; }
    S& y() { return d_[1]; }
    S& z() { return d_[2]; }
    S x() const { return d_[0]; }
    S y() const { return d_[1]; }
    S z() const { return d_[2]; }
    S* data() { return d_.data(); }
    const S* data() const { return d_.data(); }
    void setLinear(Index i, double v) { d_[i] = static_cast<S>(v); }

    // factories
    static Matrix Zero() { return Constant(S(0)); }
    static Matrix Ones() { return Constant(S(1)); }
    static Matrix Constant(S v) {
        Matrix m;
        m.setConstant(v);
        return m;
    }
    template <typename I, typename = std::enable_if_t<std::is_integral_v<I>>>
    static Matrix Zero(I n) {
        return Constant(n, S(0));
    }
    template <typename I, typename = std::enable_if_t<std::is_integral_v<I>>>
    static Matrix Ones(I n) {
        return Constant(n, S(1));
    }
    template <typename I, typename = std::enable_if_t<std::is_integral_v<I>>>
    static Matrix Constant(I n, S v) {
        Matrix m(n);
        m.setConstant(v);
        return m;
    }
    static Matrix Identity() {
        Matrix m;
        m.setIdentity();
        return m;
    }
    static Matrix UnitX() { return Matrix(S(1), S(0), S(0)); }
    static Matrix UnitY() { return Matrix(S(0), S(1), S(0)); }
    static Matrix UnitZ() { return Matrix(S(0), S(0), S(1)); }

    Matrix& setZero() { return setConstant(S(0)); }
    Matrix& setOnes() { return setConstant(S(1)); }
    Matrix& setConstant(S v) {
        std::fill(d_.begin(), d_.end(), v);
        return *this;
    }
    Matrix& setIdentity() {
        setZero();
        for (Index i = 0; i < std::min(r_, c_); ++i) (*this)(i, i) = S(1);
        return *this;
    }

    // comma initializer (m << a, b, c)
    template <typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
    shim::CommaInit<Matrix> operator<<(T v) {
        setLinear(0, static_cast<double>(v));
        return shim::CommaInit<Matrix>(*this, 1);
    }

    // compound assignment
    Matrix& operator+=(const Matrix& o) {
        for (Index i = 0; i < size(); ++i) d_[i] += o.d_[i];
        return *this;
    }
    Matrix& operator-=(const Matrix& o) {
        for (Index i = 0; i < size(); ++i) d_[i] -= o.d_[i];
        return *this;
    }
    template <typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
    Matrix& operator*=(T s) {
        for (auto& v : d_) v *= static_cast<S>(s);
        return *this;
    }
    template <typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
    Matrix& operator/=(T s) {
        for (auto& v : d_) v /= static_cast<S>(s);
        return *this;
    }

    // reductions (index order)
    S sum() const {
        S s = S(0);
        for (Index i = 0; i < size(); ++i) s = (i == 0) ? d_[0] : s + d_[i];
        return s;
    }
    S dot(const Matrix& o) const {
        S s = S(0);
        for (Index i = 0; i < size(); ++i) s = (i == 0) ? d_[0] * o.d_[0] : s + d_[i] * o.d_[i];
        return s;
    }
    S squaredNorm() const { return dot(*this); }
    S norm() const { return std::sqrt(squaredNorm()); }
    Matrix normalized() const {
        Matrix m = *this;
        S n = norm();
        if (n > S(0)) m /= n;
        return m;
    }
    void normalize() { *this = normalized(); }
    S maxCoeff() const {
        S m = d_[0];
        for (Index i = 1; i < size(); ++i)
            if (m < d_[i]) m = d_[i];
        return m;
    }
    S minCoeff() const {
        S m = d_[0];
        for (Index i = 1; i < size(); ++i)
            if (d_[i] < m) m = d_[i];
        return m;
    }
    template <int P>
    S lpNorm() const {
        if constexpr (P == Infinity) {
            S m = S(0);
            for (Index i = 0; i < size(); ++i) m = std::max(m, std::abs(d_[i]));
            return m;
        } else if constexpr (P == 1) {
            S s = S(0);
            for (Index i = 0; i < size(); ++i) s += std::abs(d_[i]);
            return s;
        } else {
            return norm();
        }
    }
    S trace() const {
        S s = S(0);
        for (Index i = 0; i < std::min(r_, c_); ++i) s = (i == 0) ? (*this)(0, 0) : s + (*this)(i, i);
        return s;
    }
    bool allFinite() const {
        for (auto v : d_)
            if (!std::isfinite(v)) return false;
        return true;
    }
    bool hasNaN() const {
        for (auto v : d_)
            if (std::isnan(v)) return true;
        return false;
    }

    // coefficient-wise
    Matrix cwiseProduct(const Matrix& o) const {
        Matrix m = *this;
        for (Index i = 0; i < size(); ++i) m.d_[i] = d_[i] * o.d_[i];
        return m;
    }
    Matrix cwiseQuotient(const Matrix& o) const {
        Matrix m = *this;
        for (Index i = 0; i < size(); ++i) m.d_[i] = d_[i] / o.d_[i];
        return m;
    }
    Matrix cwiseAbs() const {
        Matrix m = *this;
        for (auto& v : m.d_) v = std::abs(v);
        return m;
    }
    Matrix cwiseInverse() const {
        Matrix m = *this;
        for (auto& v : m.d_) v = S(1) / v;
        return m;
    }
    Matrix cwiseMax(const Matrix& o) const {
        Matrix m = *this;
        for (Index i = 0; i < size(); ++i) m.d_[i] = std::max(d_[i], o.d_[i]);
        return m;
    }
    Matrix cwiseMin(const Matrix& o) const {
        Matrix m = *this;
        for (Index i = 0; i < size(); ++i) m.d_[i] = std::min(d_[i], o.d_[i]);
        return m;
    }

    // shape
    Matrix<S, C, R> transpose() const {
        Matrix<S, C, R> t;
        if constexpr (!Matrix<S, C, R>::kFixed) t.resize(c_, r_);
        for (Index i = 0; i < r_; ++i)
            for (Index j = 0; j < c_; ++j) t(j, i) = (*this)(i, j);
        return t;
    }
    Matrix cross(const Matrix& o) const {
        return Matrix(d_[1] * o.d_[2] - d_[2] * o.d_[1], d_[2] * o.d_[0] - d_[0] * o.d_[2],
                      d_[0] * o.d_[1] - d_[1] * o.d_[0]);
    }
    S determinant() const {
        const auto& m = *this;
        return m(0, 0) * (m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1)) -
               m(0, 1) * (m(1, 0) * m(2, 2) - m(1, 2) * m(2, 0)) +
               m(0, 2) * (m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0));
    }
    // 3x3 inverse by cofactors (adjugate over the determinant)
    Matrix inverse() const {
        static_assert(R == 3 && C == 3, "inverse() is provided for 3x3 matrices");
        const auto& m = *this;
        Matrix c;
        c(0, 0) = m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1);
        c(0, 1) = m(1, 2) * m(2, 0) - m(1, 0) * m(2, 2);
        c(0, 2) = m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0);
        c(1, 0) = m(0, 2) * m(2, 1) - m(0, 1) * m(2, 2);
        c(1, 1) = m(0, 0) * m(2, 2) - m(0, 2) * m(2, 0);
        c(1, 2) = m(0, 1) * m(2, 0) - m(0, 0) * m(2, 1);
        c(2, 0) = m(0, 1) * m(1, 2) - m(0, 2) * m(1, 1);
        c(2, 1) = m(0, 2) * m(1, 0) - m(0, 0) * m(1, 2);
        c(2, 2) = m(0, 0) * m(1, 1) - m(0, 1) * m(1, 0);
        S det = m(0, 0) * c(0, 0) + m(0, 1) * c(0, 1) + m(0, 2) * c(0, 2);
        Matrix inv;
        for (Index i = 0; i < 3; ++i)
            for (Index j = 0; j < 3; ++j) inv(i, j) = c(j, i) / det;
        return inv;
    }

    // column / diagonal proxies
    class ColRef {
      public:
        ColRef(Matrix& m, Index j) : m_(m), j_(j) {}
        ColRef& operator=(const Matrix<S, R, 1>& v) {
            for (Index i = 0; i < m_.rows(); ++i) m_(i, j_) = v[i];
            return *this;
        }
        operator Matrix<S, R, 1>() const {  // NOLINT(google-explicit-constructor)
            Matrix<S, R, 1> v;
            if constexpr (!Matrix<S, R, 1>::kFixed) v.resize(m_.rows());
            for (Index i = 0; i < m_.rows(); ++i) v[i] = m_(i, j_);
            return v;
        }
        Matrix<S, R, 1> eval() const { return *this; }

      private:
        Matrix& m_;
        Index j_;
    };
    ColRef col(Index j) { return ColRef(*this, j); }
    Matrix<S, R, 1> col(Index j) const {
        Matrix<S, R, 1> v;
        if constexpr (!Matrix<S, R, 1>::kFixed) v.resize(r_);
        for (Index i = 0; i < r_; ++i) v[i] = (*this)(i, j);
        return v;
    }
    Matrix<S, 1, C> row(Index i) const {
        Matrix<S, 1, C> v;
        if constexpr (!Matrix<S, 1, C>::kFixed) v.resize(c_);
        for (Index j = 0; j < c_; ++j) v[j] = (*this)(i, j);
        return v;
    }

    class DiagRef {
      public:
        explicit DiagRef(Matrix& m) : m_(m) {}
        void setLinear(Index i, double v) { m_(i, i) = static_cast<S>(v); }
        template <typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
        shim::CommaInit<DiagRef> operator<<(T v) {
            setLinear(0, static_cast<double>(v));
            return shim::CommaInit<DiagRef>(*this, 1);
        }
        DiagRef& operator=(const Matrix<S, R, 1>& v) {
            for (Index i = 0; i < std::min(m_.rows(), m_.cols()); ++i) m_(i, i) = v[i];
            return *this;
        }
        operator Matrix<S, R, 1>() const {  // NOLINT(google-explicit-constructor)
            Matrix<S, R, 1> v;
            if constexpr (!Matrix<S, R, 1>::kFixed) v.resize(std::min(m_.rows(), m_.cols()));
            for (Index i = 0; i < std::min(m_.rows(), m_.cols()); ++i) v[i] = m_(i, i);
            return v;
        }

      private:
        Matrix& m_;
    };
    DiagRef diagonal() { return DiagRef(*this); }
    Matrix<S, R, 1> diagonal() const {
        Matrix<S, R, 1> v;
        if constexpr (!Matrix<S, R, 1>::kFixed) v.resize(std::min(r_, c_));
        for (Index i = 0; i < std::min(r_, c_); ++i) v[i] = (*this)(i, i);
        return v;
    }

    // diagonal matrix view of a vector (only used as D * x)
    struct DiagonalWrapper {
        Matrix d;
    };
    DiagonalWrapper asDiagonal() const { return DiagonalWrapper {*this}; }

    ArrayView<S, R, C> array() const;

    Matrix eval() const { return *this; }

  private:
    void alloc() {
        if constexpr (kFixed) {
            d_.fill(S(0));
        } else {
            d_.assign(static_cast<size_t>(r_ * c_), S(0));
        }
    }

    std::conditional_t<kFixed, std::array<S, (kFixed ? R * C : 1)>, std::vector<S>> d_ {};
    Index r_ = (R == Dynamic ? 0 : R);
    Index c_ = (C == Dynamic ? 0 : C);
};

// coefficient-wise array view (m.array() op n.array() / scalar)
template <typename S, int R, int C>
class ArrayView {
  public:
    explicit ArrayView(Matrix<S, R, C> m) : m_(std::move(m)) {}
    const Matrix<S, R, C>& matrix() const { return m_; }
    Matrix<S, R, C>& matrix() { return m_; }
    Index size() const { return m_.size(); }
    S operator[](Index i) const { return m_[i]; }

    template <typename F>
    ArrayView map(const ArrayView& o, F f) const {
        Matrix<S, R, C> r = m_;
        for (Index i = 0; i < size(); ++i) r[i] = f(m_[i], o.m_[i]);
        return ArrayView(std::move(r));
    }
    template <typename F>
    ArrayView mapScalar(S s, F f) const {
        Matrix<S, R, C> r = m_;
        for (Index i = 0; i < size(); ++i) r[i] = f(m_[i], s);
        return ArrayView(std::move(r));
    }
    ArrayView abs() const { return mapScalar(S(0), [](S a, S) { return std::abs(a); }); }
    ArrayView sqrt() const { return mapScalar(S(0), [](S a, S) { return std::sqrt(a); }); }
    ArrayView square() const { return mapScalar(S(0), [](S a, S) { return a * a; }); }
    ArrayView inverse() const { return mapScalar(S(0), [](S a, S) { return S(1) / a; }); }
    ArrayView max(const ArrayView& o) const { return map(o, [](S a, S b) { return std::max(a, b); }); }
    ArrayView min(const ArrayView& o) const { return map(o, [](S a, S b) { return std::min(a, b); }); }
    ArrayView max(S s) const { return mapScalar(s, [](S a, S b) { return std::max(a, b); }); }
    ArrayView min(S s) const { return mapScalar(s, [](S a, S b) { return std::min(a, b); }); }
    S sum() const { return m_.sum(); }
    S maxCoeff() const { return m_.maxCoeff(); }
    S minCoeff() const { return m_.minCoeff(); }

  private:
    Matrix<S, R, C> m_;
};

template <typename S, int R, int C>
ArrayView<S, R, C> Matrix<S, R, C>::array() const {
    return ArrayView<S, R, C>(*this);
}
template <typename S, int R, int C>
Matrix<S, R, C>::Matrix(const ArrayView<S, R, C>& a) : Matrix(a.matrix()) {}

#define PRISM_SHIM_ARRAY_OP(OP)                                                                 \
    template <typename S, int R, int C>                                                         \
    ArrayView<S, R, C> operator OP(const ArrayView<S, R, C>& a, const ArrayView<S, R, C>& b) { \
        return a.map(b, [](S x, S y) { return x OP y; });                                       \
    }                                                                                           \
    template <typename S, int R, int C, typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>> \
    ArrayView<S, R, C> operator OP(const ArrayView<S, R, C>& a, T s) {                          \
        return a.mapScalar(static_cast<S>(s), [](S x, S y) { return x OP y; });                 \
    }                                                                                           \
    template <typename S, int R, int C, typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>> \
    ArrayView<S, R, C> operator OP(T s, const ArrayView<S, R, C>& a) {                          \
        return a.mapScalar(static_cast<S>(s), [](S x, S y) { return y OP x; });                 \
    }
PRISM_SHIM_ARRAY_OP(+)
PRISM_SHIM_ARRAY_OP(-)
PRISM_SHIM_ARRAY_OP(*)
PRISM_SHIM_ARRAY_OP(/)
#undef PRISM_SHIM_ARRAY_OP

// ---- dense arithmetic
template <typename S, int R, int C>
Matrix<S, R, C> operator+(const Matrix<S, R, C>& a, const Matrix<S, R, C>& b) {
    Matrix<S, R, C> m = a;
    m += b;
    return m;
}
template <typename S, int R, int C>
Matrix<S, R, C> operator-(const Matrix<S, R, C>& a, const Matrix<S, R, C>& b) {
    Matrix<S, R, C> m = a;
    m -= b;
    return m;
}
template <typename S, int R, int C>
Matrix<S, R, C> operator-(const Matrix<S, R, C>& a) {
    Matrix<S, R, C> m = a;
    for (Index i = 0; i < m.size(); ++i) m[i] = -m[i];
    return m;
}
template <typename S, int R, int C, typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
Matrix<S, R, C> operator*(const Matrix<S, R, C>& a, T s) {
    Matrix<S, R, C> m = a;
    for (Index i = 0; i < m.size(); ++i) m[i] = a[i] * static_cast<S>(s);
    return m;
}
template <typename S, int R, int C, typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
Matrix<S, R, C> operator*(T s, const Matrix<S, R, C>& a) {
    Matrix<S, R, C> m = a;
    for (Index i = 0; i < m.size(); ++i) m[i] = static_cast<S>(s) * a[i];
    return m;
}
template <typename S, int R, int C, typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
Matrix<S, R, C> operator/(const Matrix<S, R, C>& a, T s) {
    Matrix<S, R, C> m = a;
    for (Index i = 0; i < m.size(); ++i) m[i] = a[i] / static_cast<S>(s);
    return m;
}
// matrix product, each coefficient summed over k in index order
template <typename S, int R, int K, int K2, int C>
Matrix<S, R, C> operator*(const Matrix<S, R, K>& a, const Matrix<S, K2, C>& b) {
    Matrix<S, R, C> m;
    if constexpr (!Matrix<S, R, C>::kFixed) m.resize(a.rows(), b.cols());
    for (Index i = 0; i < a.rows(); ++i)
        for (Index j = 0; j < b.cols(); ++j) {
            S s = S(0);
            for (Index k = 0; k < a.cols(); ++k) s = (k == 0) ? a(i, 0) * b(0, j) : s + a(i, k) * b(k, j);
            m(i, j) = s;
        }
    return m;
}
template <typename S, int R, int C>
bool operator==(const Matrix<S, R, C>& a, const Matrix<S, R, C>& b) {
    if (a.size() != b.size()) return false;
    for (Index i = 0; i < a.size(); ++i)
        if (!(a[i] == b[i])) return false;
    return true;
}
template <typename S, int R, int C>
bool operator!=(const Matrix<S, R, C>& a, const Matrix<S, R, C>& b) {
    return !(a == b);
}
template <typename S, int R, int C>
std::ostream& operator<<(std::ostream& os, const Matrix<S, R, C>& m) {
    for (Index i = 0; i < m.rows(); ++i) {
        for (Index j = 0; j < m.cols(); ++j) os << (j ? " " : "") << m(i, j);
        os << "\n";
    }
    return os;
}

using Vector3d = Matrix<double, 3, 1>;
using RowVector3d = Matrix<double, 1, 3>;
using Matrix3d = Matrix<double, 3, 3>;
using VectorXd = Matrix<double, Dynamic, 1>;
using RowVectorXd = Matrix<double, 1, Dynamic>;
using MatrixXd = Matrix<double, Dynamic, Dynamic>;
using MatrixX3d = Matrix<double, Dynamic, 3>;
using Vector3f = Matrix<float, 3, 1>;

// vector * diagonal-wrapper product as written in numerics/jacobi.cpp (D.asDiagonal() * r)
inline VectorXd operator*(const VectorXd::DiagonalWrapper& d, const VectorXd& x) {
    return d.d.cwiseProduct(x);
}

// ---------------------------------------------------------------- sparse
template <typename S>
class Triplet {
  public:
    Triplet() = default;
    template <typename I, typename J>
    Triplet(I i, J j, S v) : r_(static_cast<Index>(i)), c_(static_cast<Index>(j)), v_(v) {}
    Index row() const { return r_; }
    Index col() const { return c_; }
    S value() const { return v_; }

  private:
    Index r_ = 0, c_ = 0;
    S v_ = S(0);
};

// Column-major compressed sparse matrix.
template <typename S, int Options = ColMajor, typename StorageIndex = int>
class SparseMatrix {
  public:
    using Scalar = S;
    SparseMatrix() : outer_(1, 0) {}
    template <typename I, typename J>
    SparseMatrix(I rows, J cols) : rows_(static_cast<Index>(rows)), cols_(static_cast<Index>(cols)) {
        outer_.assign(static_cast<size_t>(cols_ + 1), 0);
    }

    Index rows() const { return rows_; }
    Index cols() const { return cols_; }
    Index outerSize() const { return cols_; }
    Index innerSize() const { return rows_; }
    Index nonZeros() const { return static_cast<Index>(val_.size()); }
    bool isCompressed() const { return true; }
    void makeCompressed() {}
    const StorageIndex* outerIndexPtr() const { return outer_.data(); }
    const StorageIndex* innerIndexPtr() const { return inner_.data(); }
    const S* valuePtr() const { return val_.data(); }
    S* valuePtr() { return val_.data(); }

    void resize(Index r, Index c) {
        rows_ = r;
        cols_ = c;
        setZero();
    }
    // removes every stored entry; the dimensions stay
    void setZero() {
        outer_.assign(static_cast<size_t>(cols_ + 1), 0);
        inner_.clear();
        val_.clear();
    }
    void setIdentity() {
        Index n = std::min(rows_, cols_);
        outer_.assign(static_cast<size_t>(cols_ + 1), 0);
        inner_.clear();
        val_.clear();
        for (Index j = 0; j < cols_; ++j) {
            if (j < n) {
                inner_.push_back(static_cast<StorageIndex>(j));
                val_.push_back(S(1));
            }
            outer_[j + 1] = static_cast<StorageIndex>(inner_.size());
        }
    }

    // duplicates summed in insertion order; entries sorted by row inside each column
    template <typename It>
    void setFromTriplets(It begin, It end) {
        std::vector<StorageIndex> start(static_cast<size_t>(cols_ + 1), 0);
        size_t total = 0;
        for (It it = begin; it != end; ++it) {
            Index r = it->row(), c = it->col();
            if (r < 0 || r >= rows_ || c < 0 || c >= cols_)
                throw std::out_of_range("SparseMatrix::setFromTriplets: index out of range");
            ++start[c + 1];
            ++total;
        }
        for (Index c = 0; c < cols_; ++c) start[c + 1] += start[c];
        // scatter by column, keeping the insertion order inside each column
        std::vector<StorageIndex> rows(total);
        std::vector<S> vals(total);
        std::vector<StorageIndex> fill(start.begin(), start.end() - 1);
        for (It it = begin; it != end; ++it) {
            StorageIndex p = fill[it->col()]++;
            rows[p] = static_cast<StorageIndex>(it->row());
            vals[p] = it->value();
        }
        outer_.assign(static_cast<size_t>(cols_ + 1), 0);
        inner_.clear();
        val_.clear();
        inner_.reserve(total);
        val_.reserve(total);
        std::vector<std::pair<StorageIndex, S>> col;
        for (Index c = 0; c < cols_; ++c) {
            col.assign(static_cast<size_t>(start[c + 1] - start[c]), {});
            for (StorageIndex k = start[c]; k < start[c + 1]; ++k) col[k - start[c]] = {rows[k], vals[k]};
            // stable sort by row (insertion sort: the columns of a cell matrix are short)
            for (size_t a = 1; a < col.size(); ++a) {
                auto e = col[a];
                size_t b = a;
                while (b > 0 && col[b - 1].first > e.first) {
                    col[b] = col[b - 1];
                    --b;
                }
                col[b] = e;
            }
            StorageIndex last = -1;
            for (const auto& [r, v] : col) {
                if (r == last) {
                    val_.back() = val_.back() + v;
                } else {
                    inner_.push_back(r);
                    val_.push_back(v);
                    last = r;
                }
            }
            outer_[c + 1] = static_cast<StorageIndex>(inner_.size());
        }
    }

    Index find(Index i, Index j) const {
        auto b = inner_.begin() + outer_[j], e = inner_.begin() + outer_[j + 1];
        auto it = std::lower_bound(b, e, static_cast<StorageIndex>(i));
        if (it != e && *it == i) return static_cast<Index>(it - inner_.begin());
        return -1;
    }
    S coeff(Index i, Index j) const {
        Index k = find(i, j);
        return k < 0 ? S(0) : val_[k];
    }
    // inserts a zero entry when (i, j) is not stored
    S& coeffRef(Index i, Index j) {
        Index k = find(i, j);
        if (k >= 0) return val_[k];
        auto b = inner_.begin() + outer_[j], e = inner_.begin() + outer_[j + 1];
        auto pos = std::lower_bound(b, e, static_cast<StorageIndex>(i)) - inner_.begin();
        inner_.insert(inner_.begin() + pos, static_cast<StorageIndex>(i));
        val_.insert(val_.begin() + pos, S(0));
        for (Index c = j + 1; c <= cols_; ++c) ++outer_[c];
        return val_[pos];
    }

    // union of the two patterns: a + b where both are stored, a + 0 / 0 + b elsewhere
    SparseMatrix operator+(const SparseMatrix& o) const { return combine(o, false); }
    SparseMatrix operator-(const SparseMatrix& o) const { return combine(o, true); }
    SparseMatrix& operator+=(const SparseMatrix& o) {
        *this = combine(o, false);
        return *this;
    }
    SparseMatrix& operator-=(const SparseMatrix& o) {
        *this = combine(o, true);
        return *this;
    }
    template <typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
    SparseMatrix& operator*=(T s) {
        for (auto& v : val_) v *= static_cast<S>(s);
        return *this;
    }
    template <typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
    SparseMatrix& operator/=(T s) {
        for (auto& v : val_) v /= static_cast<S>(s);
        return *this;
    }
    template <typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
    SparseMatrix operator*(T s) const {
        SparseMatrix m = *this;
        m *= s;
        return m;
    }

    // y = A x: column by column, y(i) += a_ij x_j (each row accumulated by increasing column)
    VectorXd operator*(const VectorXd& x) const {
        VectorXd y = VectorXd::Zero(rows_);
        for (Index j = 0; j < cols_; ++j) {
            S xj = x[j];
            for (StorageIndex k = outer_[j]; k < outer_[j + 1]; ++k) y[inner_[k]] += val_[k] * xj;
        }
        return y;
    }

    SparseMatrix transpose() const {
        SparseMatrix t(cols_, rows_);
        std::vector<Triplet<S>> tr;
        tr.reserve(val_.size());
        for (Index j = 0; j < cols_; ++j)
            for (StorageIndex k = outer_[j]; k < outer_[j + 1]; ++k) tr.emplace_back(j, inner_[k], val_[k]);
        t.setFromTriplets(tr.begin(), tr.end());
        return t;
    }

    // writable view of the stored diagonal entries (missing entries read as zero)
    class DiagRef {
      public:
        explicit DiagRef(SparseMatrix& m) : m_(m) {}
        Index size() const { return std::min(m_.rows(), m_.cols()); }
        S operator[](Index i) const { return m_.coeff(i, i); }
        S operator()(Index i) const { return m_.coeff(i, i); }
        operator VectorXd() const { return eval(); }  // NOLINT(google-explicit-constructor)
        VectorXd eval() const {
            VectorXd v(size());
            for (Index i = 0; i < size(); ++i) v[i] = m_.coeff(i, i);
            return v;
        }
        template <typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
        DiagRef& operator/=(T s) {
            for (Index i = 0; i < size(); ++i) {
                Index k = m_.find(i, i);
                if (k >= 0) m_.val_[k] /= static_cast<S>(s);
            }
            return *this;
        }
        template <typename T, typename = std::enable_if_t<shim::is_scalar_v<T>>>
        DiagRef& operator*=(T s) {
            for (Index i = 0; i < size(); ++i) {
                Index k = m_.find(i, i);
                if (k >= 0) m_.val_[k] *= static_cast<S>(s);
            }
            return *this;
        }
        DiagRef& operator=(const VectorXd& v) {
            for (Index i = 0; i < size(); ++i) {
                Index k = m_.find(i, i);
                if (k >= 0) m_.val_[k] = v[i];
            }
            return *this;
        }
        DiagRef& operator+=(const VectorXd& v) {
            for (Index i = 0; i < size(); ++i) {
                Index k = m_.find(i, i);
                if (k >= 0) m_.val_[k] += v[i];
            }
            return *this;
        }
        VectorXd cwiseProduct(const VectorXd& o) const { return eval().cwiseProduct(o); }
        VectorXd cwiseQuotient(const VectorXd& o) const { return eval().cwiseQuotient(o); }
        VectorXd cwiseInverse() const { return eval().cwiseInverse(); }
        VectorXd cwiseAbs() const { return eval().cwiseAbs(); }
        ArrayView<S, Dynamic, 1> array() const { return eval().array(); }
        S maxCoeff() const { return eval().maxCoeff(); }
        S minCoeff() const { return eval().minCoeff(); }
        S sum() const { return eval().sum(); }

      private:
        SparseMatrix& m_;
    };
    class ConstDiagRef {
      public:
        explicit ConstDiagRef(const SparseMatrix& m) : m_(m) {}
        Index size() const { return std::min(m_.rows(), m_.cols()); }
        S operator[](Index i) const { return m_.coeff(i, i); }
        S operator()(Index i) const { return m_.coeff(i, i); }
        operator VectorXd() const { return eval(); }  // NOLINT(google-explicit-constructor)
        VectorXd eval() const {
            VectorXd v(size());
            for (Index i = 0; i < size(); ++i) v[i] = m_.coeff(i, i);
            return v;
        }
        VectorXd cwiseProduct(const VectorXd& o) const { return eval().cwiseProduct(o); }
        VectorXd cwiseQuotient(const VectorXd& o) const { return eval().cwiseQuotient(o); }
        VectorXd cwiseInverse() const { return eval().cwiseInverse(); }
        VectorXd cwiseAbs() const { return eval().cwiseAbs(); }
        ArrayView<S, Dynamic, 1> array() const { return eval().array(); }
        S maxCoeff() const { return eval().maxCoeff(); }
        S minCoeff() const { return eval().minCoeff(); }
        S sum() const { return eval().sum(); }

      private:
        const SparseMatrix& m_;
    };
    DiagRef diagonal() { return DiagRef(*this); }
    ConstDiagRef diagonal() const { return ConstDiagRef(*this); }

  private:
    SparseMatrix combine(const SparseMatrix& o, bool minus) const {
        if (o.rows_ != rows_ || o.cols_ != cols_) throw std::invalid_argument("SparseMatrix: size mismatch");
        SparseMatrix m(rows_, cols_);
        m.inner_.reserve(inner_.size() + o.inner_.size());
        m.val_.reserve(inner_.size() + o.inner_.size());
        for (Index j = 0; j < cols_; ++j) {
            StorageIndex a = outer_[j], ae = outer_[j + 1], b = o.outer_[j], be = o.outer_[j + 1];
            while (a < ae || b < be) {
                if (a < ae && b < be && inner_[a] == o.inner_[b]) {
                    m.inner_.push_back(inner_[a]);
                    m.val_.push_back(minus ? val_[a] - o.val_[b] : val_[a] + o.val_[b]);
                    ++a;
                    ++b;
                } else if (a < ae && (b >= be || inner_[a] < o.inner_[b])) {
                    m.inner_.push_back(inner_[a]);
                    m.val_.push_back(minus ? val_[a] - S(0) : val_[a] + S(0));
                    ++a;
                } else {
                    m.inner_.push_back(o.inner_[b]);
                    m.val_.push_back(minus ? S(0) - o.val_[b] : S(0) + o.val_[b]);
                    ++b;
                }
            }
            m.outer_[j + 1] = static_cast<StorageIndex>(m.inner_.size());
        }
        return m;
    }

    Index rows_ = 0, cols_ = 0;
    std::vector<StorageIndex> outer_;
    std::vector<StorageIndex> inner_;
    std::vector<S> val_;
};

// ---------------------------------------------------------------- preconditioner and Krylov solver
namespace shim {
// row-major copy of a column-major matrix (the pattern of the reference's matrices is
// structurally symmetric, but the values are not)
struct Csr {
    Index n = 0;
    std::vector<Index> rp, ci;
    std::vector<double> v;
    template <typename M>
    void from(const M& A) {
        n = A.rows();
        rp.assign(static_cast<size_t>(n + 1), 0);
        const auto* op = A.outerIndexPtr();
        const auto* ip = A.innerIndexPtr();
        const auto* vp = A.valuePtr();
        Index nnz = A.nonZeros();
        for (Index k = 0; k < nnz; ++k) ++rp[ip[k] + 1];
        for (Index i = 0; i < n; ++i) rp[i + 1] += rp[i];
        ci.assign(static_cast<size_t>(nnz), 0);
        v.assign(static_cast<size_t>(nnz), 0.0);
        std::vector<Index> fill(rp.begin(), rp.end() - 1);
        for (Index j = 0; j < A.cols(); ++j)
            for (Index k = op[j]; k < op[j + 1]; ++k) {
                Index p = fill[ip[k]]++;
                ci[p] = j;
                v[p] = vp[k];
            }
    }
};
} // namespace shim

// Saad's ILUT: row-wise elimination with a dual threshold (entries below droptol x the
// row's 2-norm are dropped, at most fill_in entries of the row's L and of its U kept).
template <typename S>
class IncompleteLUT {
  public:
    IncompleteLUT() = default;
    void setDroptol(S d) { droptol_ = d; }
    void setFillfactor(int f) { fillfactor_ = f; }
    template <typename M>
    IncompleteLUT& compute(const M& A) {
        shim::Csr a;
        a.from(A);
        factor(a);
        return *this;
    }
    ComputationInfo info() const { return Success; }
    void solve(const std::vector<double>& b, std::vector<double>& x) const {
        x = b;
        for (Index i = 0; i < n_; ++i) {
            double s = x[i];
            for (Index q = lp_[i]; q < lp_[i + 1]; ++q) s -= lv_[q] * x[lc_[q]];
            x[i] = s;
        }
        for (Index i = n_ - 1; i >= 0; --i) {
            double s = x[i];
            for (Index q = up_[i] + 1; q < up_[i + 1]; ++q) s -= uv_[q] * x[uc_[q]];
            x[i] = s / uv_[up_[i]];
        }
    }

  private:
    void factor(const shim::Csr& A) {
        n_ = A.n;
        Index nnz = A.rp[n_];
        Index fill_in = (fillfactor_ * nnz) / std::max<Index>(n_, 1) + 1;
        lp_.assign(1, 0);
        up_.assign(1, 0);
        lc_.clear();
        lv_.clear();
        uc_.clear();
        uv_.clear();
        std::vector<double> w(static_cast<size_t>(n_), 0.0);
        std::vector<char> mark(static_cast<size_t>(n_), 0);
        std::vector<Index> L, U, done;
        for (Index i = 0; i < n_; ++i) {
            L.clear();
            U.clear();
            done.clear();
            double rownorm = 0.0;
            bool diag = false;
            for (Index k = A.rp[i]; k < A.rp[i + 1]; ++k) {
                Index j = A.ci[k];
                w[j] = A.v[k];
                mark[j] = 1;
                rownorm += A.v[k] * A.v[k];
                if (j < i) L.push_back(j);
                else if (j > i) U.push_back(j);
                else diag = true;
            }
            if (!diag) {
                w[i] = 0.0;
                mark[i] = 1;
            }
            rownorm = std::sqrt(rownorm);
            // eliminate the lower part in increasing column order (fill joins the list)
            while (!L.empty()) {
                size_t pos = 0;
                for (size_t q = 1; q < L.size(); ++q)
                    if (L[q] < L[pos]) pos = q;
                Index k = L[pos];
                L[pos] = L.back();
                L.pop_back();
                double fact = w[k] / uv_[up_[k]];
                if (std::abs(fact) <= droptol_ * rownorm) {
                    w[k] = 0.0;
                    mark[k] = 0;
                    continue;
                }
                w[k] = fact;
                done.push_back(k);
                for (Index q = up_[k] + 1; q < up_[k + 1]; ++q) {
                    Index j = uc_[q];
                    if (!mark[j]) {
                        mark[j] = 1;
                        w[j] = 0.0;
                        if (j < i) L.push_back(j);
                        else if (j > i) U.push_back(j);
                    }
                    w[j] -= fact * uv_[q];
                }
            }
            auto keep = [&](std::vector<Index>& idx) {
                std::vector<Index> kept;
                for (auto j : idx)
                    if (std::abs(w[j]) > droptol_ * rownorm) kept.push_back(j);
                if (static_cast<Index>(kept.size()) > fill_in) {
                    std::nth_element(kept.begin(), kept.begin() + fill_in, kept.end(),
                                     [&](Index a, Index b) { return std::abs(w[a]) > std::abs(w[b]); });
                    kept.resize(static_cast<size_t>(fill_in));
                }
                std::sort(kept.begin(), kept.end());
                return kept;
            };
            auto Lk = keep(done);
            auto Uk = keep(U);
            for (auto j : Lk) {
                lc_.push_back(j);
                lv_.push_back(w[j]);
            }
            lp_.push_back(static_cast<Index>(lc_.size()));
            double d = w[i];
            if (d == 0.0) d = (0.0001 + droptol_) * rownorm;
            uc_.push_back(i);
            uv_.push_back(d);
            for (auto j : Uk) {
                uc_.push_back(j);
                uv_.push_back(w[j]);
            }
            up_.push_back(static_cast<Index>(uc_.size()));
            for (auto j : done) {
                w[j] = 0.0;
                mark[j] = 0;
            }
            for (auto j : U) {
                w[j] = 0.0;
                mark[j] = 0;
            }
            for (Index k = A.rp[i]; k < A.rp[i + 1]; ++k) {
                w[A.ci[k]] = 0.0;
                mark[A.ci[k]] = 0;
            }
            w[i] = 0.0;
            mark[i] = 0;
        }
    }

    S droptol_ = NumTraits<S>::dummy_precision();
    int fillfactor_ = 10;
    Index n_ = 0;
    std::vector<Index> lp_, lc_, up_, uc_;
    std::vector<double> lv_, uv_;
};

template <typename S>
class DiagonalPreconditioner {
  public:
    template <typename M>
    DiagonalPreconditioner& compute(const M& A) {
        VectorXd d = A.diagonal();
        inv_.assign(static_cast<size_t>(d.size()), 1.0);
        for (Index i = 0; i < d.size(); ++i) inv_[i] = d[i] != 0 ? 1.0 / d[i] : 1.0;
        return *this;
    }
    void solve(const std::vector<double>& b, std::vector<double>& x) const {
        x.resize(b.size());
        for (size_t i = 0; i < b.size(); ++i) x[i] = inv_[i] * b[i];
    }

  private:
    std::vector<double> inv_;
};

template <typename M, typename P = DiagonalPreconditioner<typename M::Scalar>>
class BiCGSTAB {
  public:
    BiCGSTAB() = default;
    BiCGSTAB& compute(const M& A) {
        a_.from(A);
        pre_.compute(A);
        return *this;
    }
    void setTolerance(double t) { tol_ = t; }
    void setMaxIterations(Index m) { max_iters_ = m; }
    double tolerance() const { return tol_; }
    Index maxIterations() const { return max_iters_ < 0 ? 2 * a_.n : max_iters_; }
    Index iterations() const { return iters_; }
    double error() const { return error_; }
    ComputationInfo info() const { return info_; }
    P& preconditioner() { return pre_; }

    VectorXd solve(const VectorXd& b) const { return solveWithGuess(b, VectorXd::Zero(b.size())); }

    VectorXd solveWithGuess(const VectorXd& bb, const VectorXd& x0) const {
        const Index n = a_.n;
        std::vector<double> b(bb.data(), bb.data() + n), x(x0.data(), x0.data() + n);
        run(b, x);
        VectorXd out(n);
        for (Index i = 0; i < n; ++i) out[i] = x[i];
        return out;
    }

  private:
    void spmv(const std::vector<double>& x, std::vector<double>& y) const {
        y.assign(static_cast<size_t>(a_.n), 0.0);
        for (Index i = 0; i < a_.n; ++i) {
            double s = 0.0;
            for (Index k = a_.rp[i]; k < a_.rp[i + 1]; ++k) s += a_.v[k] * x[a_.ci[k]];
            y[i] = s;
        }
    }
    static double vdot(const std::vector<double>& a, const std::vector<double>& b) {
        double s = 0.0;
        for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
        return s;
    }
    void run(const std::vector<double>& b, std::vector<double>& x) const {
        const Index n = a_.n;
        const double eps = NumTraits<double>::epsilon();
        const Index maxIters = maxIterations();
        std::vector<double> r(n), r0, Ax;
        spmv(x, Ax);
        for (Index i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
        r0 = r;
        double r0_sqnorm = vdot(r0, r0);
        double rhs_sqnorm = vdot(b, b);
        iters_ = 0;
        info_ = Success;
        if (rhs_sqnorm == 0) {
            std::fill(x.begin(), x.end(), 0.0);
            error_ = 0;
            return;
        }
        double rho = 1, alpha = 1, w = 1;
        std::vector<double> v(n, 0.0), p(n, 0.0), y(n), z(n), s(n), t(n);
        const double tol2 = tol_ * tol_ * rhs_sqnorm;
        const double eps2 = eps * eps;
        Index i = 0, restarts = 0;
        while (vdot(r, r) > tol2 && i < maxIters) {
            double rho_old = rho;
            rho = vdot(r0, r);
            if (std::abs(rho) < eps2 * r0_sqnorm) {
                // r0 is almost orthogonal to r: restart from the current residual
                spmv(x, Ax);
                for (Index k = 0; k < n; ++k) r[k] = b[k] - Ax[k];
                r0 = r;
                rho = r0_sqnorm = vdot(r, r);
                if (restarts++ == 0) i = 0;
            }
            double beta = (rho / rho_old) * (alpha / w);
            for (Index k = 0; k < n; ++k) p[k] = r[k] + beta * (p[k] - w * v[k]);
            pre_.solve(p, y);
            spmv(y, v);
            alpha = rho / vdot(r0, v);
            for (Index k = 0; k < n; ++k) s[k] = r[k] - alpha * v[k];
            pre_.solve(s, z);
            spmv(z, t);
            double tmp = vdot(t, t);
            w = tmp > 0.0 ? vdot(t, s) / tmp : 0.0;
            for (Index k = 0; k < n; ++k) x[k] += alpha * y[k] + w * z[k];
            for (Index k = 0; k < n; ++k) r[k] = s[k] - w * t[k];
            ++i;
        }
        iters_ = i;
        error_ = std::sqrt(vdot(r, r) / rhs_sqnorm);
        info_ = (vdot(r, r) > tol2) ? NoConvergence : Success;
    }

    shim::Csr a_;
    P pre_;
    double tol_ = NumTraits<double>::epsilon();
    Index max_iters_ = -1;
    mutable Index iters_ = 0;
    mutable double error_ = 0;
    mutable ComputationInfo info_ = Success;
};

} // namespace Eigen
