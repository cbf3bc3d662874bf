// Minimal stand-in for the subset of the Eigen 3.4 public API that the
// reference's CCD sources use (fixed-size vectors/matrices, AlignedBox,
// aligned_allocator).  It exists ONLY so that the reference's own, unmodified
// BVHTree.cpp / BVHLeaf.cpp / NarrowPhase.cpp / CTCD.cpp can be compiled into
// the test oracle; it is test infrastructure and never part of the product.
//
// Written from Eigen's documented API semantics, not from Eigen's sources.
// Arithmetic follows the evaluation order that Eigen produces for the small
// fixed-size vectors the reference uses:
//   * coefficient-wise expressions are evaluated per coefficient, left to right
//     exactly as written (a + b*s + c*t  ->  (a_k + b_k*s) + c_k*t);
//   * reductions (dot, squaredNorm, sum) accumulate left to right:
//     ((x0 + x1) + x2) + x3.  For sizes 2 and 3 this equals Eigen's packet
//     reduction on SSE2/AVX (one 2-lane packet reduced, then the tail added).
//   * norm() = sqrt(squaredNorm()).
#pragma once

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <functional>
#include <string>
#include <initializer_list>
#include <limits>
#include <memory>
#include <type_traits>
#include <vector>

#define EIGEN_MAKE_ALIGNED_OPERATOR_NEW_IF_VECTORIZABLE_FIXED_SIZE(Scalar, Dim)
#define EIGEN_MAKE_ALIGNED_OPERATOR_NEW
#define EIGEN_STRONG_INLINE inline
#ifndef eigen_assert
#define eigen_assert(x) assert(x)
#endif

namespace Eigen {

const int Dynamic = -1;
enum StorageOptions { ColMajor = 0, RowMajor = 0x1, AutoAlign = 0, DontAlign = 0x2 };

template <typename T>
using aligned_allocator = std::allocator<T>;

// Only ever named by the reference in member templates it does not
// instantiate (the Eigen-matrix convenience overloads of update/traverse).
template <typename Derived>
class MatrixBase;

template <typename T, int R, int C, int Opt = 0, int MR = R, int MC = C>
class Matrix;

namespace mini {

// Coefficient-wise view used by .array(): supports the in-place scalar
// updates the reference performs (box.min().array() -= eta).
template <typename M>
class ArrayRef {
public:
    explicit ArrayRef(M &m) : m_(m) {}
    template <typename S> ArrayRef &operator+=(const S &s) { for (int i = 0; i < M::SizeAtCompileTime; ++i) m_[i] += s; return *this; }
    template <typename S> ArrayRef &operator-=(const S &s) { for (int i = 0; i < M::SizeAtCompileTime; ++i) m_[i] -= s; return *this; }
    template <typename S> ArrayRef &operator*=(const S &s) { for (int i = 0; i < M::SizeAtCompileTime; ++i) m_[i] *= s; return *this; }
    template <typename S> ArrayRef &operator/=(const S &s) { for (int i = 0; i < M::SizeAtCompileTime; ++i) m_[i] /= s; return *this; }
private:
    M &m_;
};

// Writable column of a fixed-size matrix (Matrix2d::col(j) = v).
template <typename T, int R, int C, int Opt, int MR, int MC>
class ColRef {
public:
    ColRef(Matrix<T, R, C, Opt, MR, MC> &m, int j) : m_(m), j_(j) {}
    template <int R2, int C2, int O2, int MR2, int MC2>
    ColRef &operator=(const Matrix<T, R2, C2, O2, MR2, MC2> &v)
    {
        static_assert(R2 * C2 == R, "column size mismatch");
        for (int i = 0; i < R; ++i) m_(i, j_) = v[i];
        return *this;
    }
    operator Matrix<T, R, 1>() const
    {
        Matrix<T, R, 1> out;
        for (int i = 0; i < R; ++i) out[i] = m_(i, j_);
        return out;
    }
    T operator[](int i) const { return m_(i, j_); }
private:
    Matrix<T, R, C, Opt, MR, MC> &m_;
    int j_;
};

} // namespace mini

// Fixed-size dense matrix, column-major storage.
template <typename T, int R, int C, int Opt, int MR, int MC>
class Matrix {
    static_assert(R > 0 && C > 0, "only fixed sizes are provided by this stand-in");
public:
    typedef T Scalar;
    typedef T RealScalar;
    enum { RowsAtCompileTime = R, ColsAtCompileTime = C, SizeAtCompileTime = R * C };

    Matrix() { for (int i = 0; i < R * C; ++i) d_[i] = T(0); }
    Matrix(const T &x, const T &y) { static_assert(R * C == 2, "size"); d_[0] = x; d_[1] = y; }
    Matrix(const T &x, const T &y, const T &z) { static_assert(R * C == 3, "size"); d_[0] = x; d_[1] = y; d_[2] = z; }
    Matrix(const T &x, const T &y, const T &z, const T &w) { static_assert(R * C == 4, "size"); d_[0] = x; d_[1] = y; d_[2] = z; d_[3] = w; }
    Matrix(const Matrix &o) = default;
    Matrix &operator=(const Matrix &o) = default;

    // Vectors convert between row and column orientation (Eigen allows
    // assigning a column vector to a row vector of the same size).
    template <int R2, int C2, int O2, int MR2, int MC2,
              typename = typename std::enable_if<(R2 != R || C2 != C) && R2 * C2 == R * C &&
                                                 (R == 1 || C == 1) && (R2 == 1 || C2 == 1)>::type>
    Matrix(const Matrix<T, R2, C2, O2, MR2, MC2> &o) { for (int i = 0; i < R * C; ++i) d_[i] = o[i]; }
    template <int O2, int MR2, int MC2, typename = typename std::enable_if<O2 != Opt || MR2 != MR || MC2 != MC>::type>
    Matrix(const Matrix<T, R, C, O2, MR2, MC2> &o) { for (int i = 0; i < R * C; ++i) d_[i] = o[i]; }
    Matrix(const mini::ColRef<T, R, C, Opt, MR, MC> &) = delete;

    static int rows() { return R; }
    static int cols() { return C; }
    static int size() { return R * C; }

    T &operator[](int i) { return d_[i]; }
    const T &operator[](int i) const { return d_[i]; }
    T &operator()(int i) { return d_[i]; }
    const T &operator()(int i) const { return d_[i]; }
    T &operator()(int i, int j) { return d_[j * R + i]; }
    const T &operator()(int i, int j) const { return d_[j * R + i]; }
    T *data() { return d_; }
    const T *data() const { return d_; }

    static Matrix Zero() { return Constant(T(0)); }
    static Matrix Ones() { return Constant(T(1)); }
    static Matrix Constant(const T &v) { Matrix m; m.setConstant(v); return m; }
    Matrix &setZero() { return setConstant(T(0)); }
    Matrix &setOnes() { return setConstant(T(1)); }
    Matrix &setConstant(const T &v) { for (int i = 0; i < R * C; ++i) d_[i] = v; return *this; }

    Matrix operator+(const Matrix &o) const { Matrix r; for (int i = 0; i < R * C; ++i) r.d_[i] = d_[i] + o.d_[i]; return r; }
    Matrix operator-(const Matrix &o) const { Matrix r; for (int i = 0; i < R * C; ++i) r.d_[i] = d_[i] - o.d_[i]; return r; }
    Matrix operator-() const { Matrix r; for (int i = 0; i < R * C; ++i) r.d_[i] = -d_[i]; return r; }
    Matrix operator*(const T &s) const { Matrix r; for (int i = 0; i < R * C; ++i) r.d_[i] = d_[i] * s; return r; }
    Matrix operator/(const T &s) const { Matrix r; for (int i = 0; i < R * C; ++i) r.d_[i] = d_[i] / s; return r; }
    Matrix &operator+=(const Matrix &o) { for (int i = 0; i < R * C; ++i) d_[i] += o.d_[i]; return *this; }
    Matrix &operator-=(const Matrix &o) { for (int i = 0; i < R * C; ++i) d_[i] -= o.d_[i]; return *this; }
    Matrix &operator*=(const T &s) { for (int i = 0; i < R * C; ++i) d_[i] *= s; return *this; }
    Matrix &operator/=(const T &s) { for (int i = 0; i < R * C; ++i) d_[i] /= s; return *this; }
    bool operator==(const Matrix &o) const { for (int i = 0; i < R * C; ++i) if (!(d_[i] == o.d_[i])) return false; return true; }
    bool operator!=(const Matrix &o) const { return !(*this == o); }

    T dot(const Matrix &o) const { T s = d_[0] * o.d_[0]; for (int i = 1; i < R * C; ++i) s = s + d_[i] * o.d_[i]; return s; }
    T squaredNorm() const { return dot(*this); }
    T norm() const { using std::sqrt; return sqrt(squaredNorm()); }
    T sum() const { T s = d_[0]; for (int i = 1; i < R * C; ++i) s = s + d_[i]; return s; }
    T maxCoeff() const { T m = d_[0]; for (int i = 1; i < R * C; ++i) m = (m < d_[i]) ? d_[i] : m; return m; }
    T minCoeff() const { T m = d_[0]; for (int i = 1; i < R * C; ++i) m = (d_[i] < m) ? d_[i] : m; return m; }
    Matrix cwiseMin(const Matrix &o) const { Matrix r; for (int i = 0; i < R * C; ++i) r.d_[i] = (o.d_[i] < d_[i]) ? o.d_[i] : d_[i]; return r; }
    Matrix cwiseMax(const Matrix &o) const { Matrix r; for (int i = 0; i < R * C; ++i) r.d_[i] = (d_[i] < o.d_[i]) ? o.d_[i] : d_[i]; return r; }
    Matrix cwiseAbs() const { using std::abs; Matrix r; for (int i = 0; i < R * C; ++i) r.d_[i] = abs(d_[i]); return r; }

    Matrix cross(const Matrix &b) const
    {
        static_assert(R * C == 3, "cross needs 3-vectors");
        return Matrix(d_[1] * b.d_[2] - d_[2] * b.d_[1],
                      d_[2] * b.d_[0] - d_[0] * b.d_[2],
                      d_[0] * b.d_[1] - d_[1] * b.d_[0]);
    }
    void normalize() { T z = squaredNorm(); if (z > T(0)) { using std::sqrt; *this /= sqrt(z); } }
    Matrix normalized() const { Matrix r(*this); r.normalize(); return r; }
    // Scales by the largest magnitude first so that tiny or huge vectors do
    // not under/overflow while being normalised.
    void stableNormalize()
    {
        T w = cwiseAbs().maxCoeff();
        if (w > T(0)) {
            Matrix s = *this / w;
            T z = s.squaredNorm();
            using std::sqrt;
            if (z > T(0)) *this = s / sqrt(z);
        }
    }
    Matrix stableNormalized() const { Matrix r(*this); r.stableNormalize(); return r; }

    T determinant() const
    {
        static_assert(R == C && (R == 2 || R == 3), "determinant for 2x2 / 3x3 only");
        const Matrix &m = *this;
        if (R == 2) return m(0, 0) * m(1, 1) - m(1, 0) * m(0, 1);
        return m(0, 0) * (m(1 % R, 1 % C) * m(2 % R, 2 % C) - m(2 % R, 1 % C) * m(1 % R, 2 % C))
             - m(1 % R, 0) * (m(0, 1 % C) * m(2 % R, 2 % C) - m(2 % R, 1 % C) * m(0, 2 % C))
             + m(2 % R, 0) * (m(0, 1 % C) * m(1 % R, 2 % C) - m(1 % R, 1 % C) * m(0, 2 % C));
    }

    template <int N>
    Matrix<T, N, 1> head() const
    {
        // The reference names head<3>() on 2-vectors inside branches that are
        // never taken for DIM==2; it must compile, and copies what exists.
        Matrix<T, N, 1> r;
        for (int i = 0; i < N && i < R * C; ++i) r[i] = d_[i];
        return r;
    }
    template <typename U>
    Matrix<U, R, C, Opt, MR, MC> cast() const { Matrix<U, R, C, Opt, MR, MC> r; for (int i = 0; i < R * C; ++i) r[i] = U(d_[i]); return r; }

    mini::ColRef<T, R, C, Opt, MR, MC> col(int j) { return mini::ColRef<T, R, C, Opt, MR, MC>(*this, j); }
    Matrix<T, R, 1> col(int j) const { Matrix<T, R, 1> r; for (int i = 0; i < R; ++i) r[i] = (*this)(i, j); return r; }
    mini::ArrayRef<Matrix> array() { return mini::ArrayRef<Matrix>(*this); }

private:
    T d_[R * C];
};

template <typename T, int R, int C, int Opt, int MR, int MC>
inline Matrix<T, R, C, Opt, MR, MC> operator*(const T &s, const Matrix<T, R, C, Opt, MR, MC> &m)
{
    Matrix<T, R, C, Opt, MR, MC> r;
    for (int i = 0; i < R * C; ++i) r[i] = s * m[i];
    return r;
}

// Dynamic-row matrices (VectorXi, and the RowMajor copies named by the
// reference's Eigen convenience overloads): only storage and shape queries.
template <typename T, int C, int Opt, int MR, int MC>
class Matrix<T, Dynamic, C, Opt, MR, MC> {
public:
    typedef T Scalar;
    Matrix() : r_(0), c_(C == Dynamic ? 0 : C) {}
    explicit Matrix(int n) : v_(std::size_t(n) * (C == Dynamic ? 1 : C)), r_(n), c_(C == Dynamic ? 1 : C) {}
    Matrix(int r, int c) : v_(std::size_t(r) * c), r_(r), c_(c) {}
    int size() const { return int(v_.size()); }
    int rows() const { return r_; }
    int cols() const { return c_; }
    T *data() { return v_.data(); }
    const T *data() const { return v_.data(); }
    T &operator[](int i) { return v_[i]; }
    const T &operator[](int i) const { return v_[i]; }
    T &operator()(int i) { return v_[i]; }
    const T &operator()(int i) const { return v_[i]; }
    T &operator()(int i, int j) { return (Opt & RowMajor) ? v_[std::size_t(i) * c_ + j] : v_[std::size_t(j) * r_ + i]; }
    const T &operator()(int i, int j) const { return (Opt & RowMajor) ? v_[std::size_t(i) * c_ + j] : v_[std::size_t(j) * r_ + i]; }
private:
    std::vector<T> v_;
    int r_, c_;
};

typedef Matrix<double, 2, 1> Vector2d;
typedef Matrix<double, 3, 1> Vector3d;
typedef Matrix<double, 4, 1> Vector4d;
typedef Matrix<float, 2, 1> Vector2f;
typedef Matrix<float, 3, 1> Vector3f;
typedef Matrix<float, 4, 1> Vector4f;
typedef Matrix<int, 2, 1> Vector2i;
typedef Matrix<int, 3, 1> Vector3i;
typedef Matrix<int, 4, 1> Vector4i;
typedef Matrix<double, 2, 2> Matrix2d;
typedef Matrix<double, 3, 3> Matrix3d;
typedef Matrix<double, 1, 3> RowVector3d;
typedef Matrix<int, Dynamic, 1> VectorXi;
typedef Matrix<double, Dynamic, 1> VectorXd;

// Axis-aligned box.  Empty boxes have min = +highest, max = lowest; a box is
// empty when any min exceeds the matching max.  Boxes are closed sets.
template <typename T, int D>
class AlignedBox {
public:
    typedef T Scalar;
    typedef Matrix<T, D, 1> VectorType;
    enum { AmbientDimAtCompileTime = D };

    AlignedBox() { setEmpty(); }
    AlignedBox(const VectorType &a, const VectorType &b) : min_(a), max_(b) {}
    virtual ~AlignedBox() {}

    VectorType &min() { return min_; }
    const VectorType &min() const { return min_; }
    VectorType &max() { return max_; }
    const VectorType &max() const { return max_; }

    void setEmpty()
    {
        min_.setConstant(std::numeric_limits<T>::max());
        max_.setConstant(std::numeric_limits<T>::lowest());
    }
    bool isEmpty() const
    {
        for (int i = 0; i < D; ++i) if (!(min_[i] <= max_[i])) return true;
        return false;
    }
    AlignedBox &extend(const VectorType &p)
    {
        min_ = min_.cwiseMin(p);
        max_ = max_.cwiseMax(p);
        return *this;
    }
    AlignedBox &extend(const AlignedBox &b)
    {
        min_ = min_.cwiseMin(b.min_);
        max_ = max_.cwiseMax(b.max_);
        return *this;
    }
    bool intersects(const AlignedBox &b) const
    {
        for (int i = 0; i < D; ++i) {
            T lo = (min_[i] < b.min_[i]) ? b.min_[i] : min_[i];
            T hi = (b.max_[i] < max_[i]) ? b.max_[i] : max_[i];
            if (!(lo <= hi)) return false;
        }
        return true;
    }
    bool contains(const VectorType &p) const
    {
        for (int i = 0; i < D; ++i) if (!(min_[i] <= p[i] && p[i] <= max_[i])) return false;
        return true;
    }
    bool contains(const AlignedBox &b) const { return contains(b.min_) && contains(b.max_); }
    VectorType center() const { return (min_ + max_) / T(2); }
    VectorType sizes() const { return max_ - min_; }

protected:
    VectorType min_, max_;
};

} // namespace Eigen
