// zynum/matrix_multiply.hpp — C++ mirror of Zynum's checked, typed GEMM API.
//
// Mirrors src/blas/api/operations.zig:501 matrixMultiply and :529
// matrixMultiplyWithWorkspace, with the views and error set of
// src/blas/api/views.zig (ConstMatrix / Matrix, Error :22-30,
// requiredMatrixStorageLength, MatrixTransform normal / transposed / adjoint)
// and the overlap checks of src/blas/api/aliasing.zig.  The product itself
// runs on the GPU through the Fortran ABI of libzynum_blas_gpu.so
// (dgemm_ / sgemm_ / zgemm_ / cgemm_).  Header-only; link -lzynum_blas_gpu.
#pragma once

#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#include "../zynum_blas_gpu.h"

namespace zynum {

using BlasInt = int32_t;

// views.zig:22-30
enum class Error : int {
    None = 0,
    DimensionMismatch,
    InvalidLength,
    InvalidStride,
    InvalidLeadingDimension,
    BufferTooSmall,
    WorkspaceTooSmall,
    AliasingNotAllowed,
};

// views.zig MatrixTransform
enum class MatrixTransform { normal, transposed, adjoint };

// views.zig requiredMatrixStorageLength
inline Error required_matrix_storage(BlasInt rows, BlasInt cols, BlasInt ld, size_t* out) {
    if (rows < 0 || cols < 0) return Error::InvalidLength;
    if (rows == 0 || cols == 0) {
        *out = 0;
        return Error::None;
    }
    if (ld < (rows > 1 ? rows : 1)) return Error::InvalidLeadingDimension;
    *out = (size_t)rows + (size_t)(cols - 1) * (size_t)ld;
    return Error::None;
}

template <typename T>
struct ConstMatrix {
    const T* values = nullptr;
    size_t length = 0;  // elements available behind `values`
    BlasInt row_count = 0, column_count = 0, leading_dimension = 1;
    MatrixTransform operation = MatrixTransform::normal;

    ConstMatrix transposed() const {
        ConstMatrix m = *this;
        m.operation = operation == MatrixTransform::normal ? MatrixTransform::transposed : MatrixTransform::normal;
        return m;
    }
    ConstMatrix adjoint() const {
        ConstMatrix m = *this;
        m.operation = operation == MatrixTransform::normal ? MatrixTransform::adjoint : MatrixTransform::normal;
        return m;
    }
    BlasInt effective_row_count() const { return operation == MatrixTransform::normal ? row_count : column_count; }
    BlasInt effective_column_count() const { return operation == MatrixTransform::normal ? column_count : row_count; }
    Error check() const {
        size_t need = 0;
        Error e = required_matrix_storage(row_count, column_count, leading_dimension, &need);
        if (e != Error::None) return e;
        return need > length ? Error::BufferTooSmall : Error::None;
    }
};

template <typename T>
struct Matrix {
    T* values = nullptr;
    size_t length = 0;
    BlasInt row_count = 0, column_count = 0, leading_dimension = 1;

    ConstMatrix<T> as_const() const {
        return {values, length, row_count, column_count, leading_dimension, MatrixTransform::normal};
    }
    Error check() const { return as_const().check(); }
};

// views.zig:171 constMatrix / :189 matrix (leading dimension defaults to row_count)
template <typename T>
Error const_matrix(const T* values, size_t length, BlasInt rows, BlasInt cols, ConstMatrix<T>* out,
                   BlasInt ld = -1) {
    ConstMatrix<T> m{values, length, rows, cols, ld < 0 ? rows : ld, MatrixTransform::normal};
    Error e = m.check();
    if (e == Error::None) *out = m;
    return e;
}
template <typename T>
Error matrix(T* values, size_t length, BlasInt rows, BlasInt cols, Matrix<T>* out, BlasInt ld = -1) {
    Matrix<T> m{values, length, rows, cols, ld < 0 ? rows : ld};
    Error e = m.check();
    if (e == Error::None) *out = m;
    return e;
}

namespace detail {
template <typename T>
bool overlaps(const void* a, size_t an, const void* b, size_t bn) {
    if (an == 0 || bn == 0) return false;
    const char* a0 = static_cast<const char*>(a);
    const char* b0 = static_cast<const char*>(b);
    return a0 < b0 + bn * sizeof(T) && b0 < a0 + an * sizeof(T);
}
template <typename T>
size_t span(const ConstMatrix<T>& m) {
    size_t n = 0;
    required_matrix_storage(m.row_count, m.column_count, m.leading_dimension, &n);
    return n;
}
inline char trans_char(MatrixTransform t) {
    return t == MatrixTransform::normal ? 'N' : (t == MatrixTransform::transposed ? 'T' : 'C');
}
inline void gemm(char ta, char tb, BlasInt m, BlasInt n, BlasInt k, double al, const double* a, BlasInt lda,
                 const double* b, BlasInt ldb, double be, double* c, BlasInt ldc) {
    dgemm_(&ta, &tb, &m, &n, &k, &al, a, &lda, b, &ldb, &be, c, &ldc);
}
inline void gemm(char ta, char tb, BlasInt m, BlasInt n, BlasInt k, float al, const float* a, BlasInt lda,
                 const float* b, BlasInt ldb, float be, float* c, BlasInt ldc) {
    sgemm_(&ta, &tb, &m, &n, &k, &al, a, &lda, b, &ldb, &be, c, &ldc);
}
inline void gemm(char ta, char tb, BlasInt m, BlasInt n, BlasInt k, std::complex<double> al,
                 const std::complex<double>* a, BlasInt lda, const std::complex<double>* b, BlasInt ldb,
                 std::complex<double> be, std::complex<double>* c, BlasInt ldc) {
    zgemm_(&ta, &tb, &m, &n, &k, &al, a, &lda, b, &ldb, &be, c, &ldc);
}
inline void gemm(char ta, char tb, BlasInt m, BlasInt n, BlasInt k, std::complex<float> al,
                 const std::complex<float>* a, BlasInt lda, const std::complex<float>* b, BlasInt ldb,
                 std::complex<float> be, std::complex<float>* c, BlasInt ldc) {
    cgemm_(&ta, &tb, &m, &n, &k, &al, a, &lda, b, &ldb, &be, c, &ldc);
}

// operations.zig:139 checkMatrixProductShapes
template <typename T>
Error check_shapes(const ConstMatrix<T>& l, const ConstMatrix<T>& r, const Matrix<T>& out) {
    if (l.effective_column_count() != r.effective_row_count()) return Error::DimensionMismatch;
    if (out.row_count != l.effective_row_count()) return Error::DimensionMismatch;
    if (out.column_count != r.effective_column_count()) return Error::DimensionMismatch;
    return Error::None;
}
}  // namespace detail

// result = product_scale * op(left) * op(right) + result_scale * result
// (operations.zig:501; product_scale defaults to 1, result_scale to 0).
template <typename T>
Error matrix_multiply(const ConstMatrix<T>& left, const ConstMatrix<T>& right, const Matrix<T>& result,
                      T product_scale = T(1), T result_scale = T(0)) {
    Error e;
    if ((e = left.check()) != Error::None || (e = right.check()) != Error::None || (e = result.check()) != Error::None)
        return e;
    if ((e = detail::check_shapes(left, right, result)) != Error::None) return e;
    const size_t rn = detail::span(result.as_const());
    if (detail::overlaps<T>(result.values, rn, left.values, detail::span(left)) ||
        detail::overlaps<T>(result.values, rn, right.values, detail::span(right)))
        return Error::AliasingNotAllowed;
    if (result.row_count == 0 || result.column_count == 0) return Error::None;
    detail::gemm(detail::trans_char(left.operation), detail::trans_char(right.operation), result.row_count,
                 result.column_count, left.effective_column_count(), product_scale, left.values,
                 left.leading_dimension, right.values, right.leading_dimension, result_scale, result.values,
                 result.leading_dimension);
    return Error::None;
}

// Workspace length of matrixMultiplyWithWorkspace: row_count x column_count.
template <typename T>
size_t matrix_multiply_workspace_length(const Matrix<T>& result) {
    return (size_t)(result.row_count > 0 ? result.row_count : 0) *
           (size_t)(result.column_count > 0 ? result.column_count : 0);
}

// Caller-approved aliasing of the result with an input (operations.zig:529):
// the product goes to `workspace` and is copied back.
template <typename T>
Error matrix_multiply_with_workspace(const ConstMatrix<T>& left, const ConstMatrix<T>& right, const Matrix<T>& result,
                                     T* workspace, size_t workspace_length, T product_scale = T(1),
                                     T result_scale = T(0)) {
    Error e;
    if ((e = left.check()) != Error::None || (e = right.check()) != Error::None || (e = result.check()) != Error::None)
        return e;
    if ((e = detail::check_shapes(left, right, result)) != Error::None) return e;
    const size_t need = matrix_multiply_workspace_length(result);
    if (workspace_length < need) return Error::WorkspaceTooSmall;
    if (detail::overlaps<T>(workspace, need, left.values, detail::span(left)) ||
        detail::overlaps<T>(workspace, need, right.values, detail::span(right)) ||
        detail::overlaps<T>(workspace, need, result.values, detail::span(result.as_const())))
        return Error::AliasingNotAllowed;
    if (need == 0) return Error::None;
    const BlasInt m = result.row_count, n = result.column_count;
    for (BlasInt j = 0; j < n; ++j)
        for (BlasInt i = 0; i < m; ++i) workspace[i + (size_t)j * m] = result.values[i + (size_t)j * result.leading_dimension];
    detail::gemm(detail::trans_char(left.operation), detail::trans_char(right.operation), m, n,
                 left.effective_column_count(), product_scale, left.values, left.leading_dimension, right.values,
                 right.leading_dimension, result_scale, workspace, m);
    for (BlasInt j = 0; j < n; ++j)
        for (BlasInt i = 0; i < m; ++i) result.values[i + (size_t)j * result.leading_dimension] = workspace[i + (size_t)j * m];
    return Error::None;
}

}  // namespace zynum
