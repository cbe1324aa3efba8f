// Typed API (zynum/matrix_multiply.hpp) tests, following test/api/zynum_test.zig:28-158.
//   typed_api_test checks   argument / shape / aliasing errors (no GPU work)
//   typed_api_test compute  products through libzynum_blas_gpu.so (needs a GPU)
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>

#include "zynum/matrix_multiply.hpp"

using zynum::Error;

static int failures = 0;
#define EXPECT(cond)                                                \
    do {                                                            \
        if (!(cond)) {                                              \
            std::fprintf(stderr, "FAILED %s:%d %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                             \
        }                                                           \
    } while (0)

static void checks() {
    // zynum_test.zig:57-78: structural errors
    double m4[4] = {1, 2, 3, 4};
    zynum::ConstMatrix<double> v;
    EXPECT(zynum::const_matrix(m4, 4, 2, 2, &v, 1) == Error::InvalidLeadingDimension);
    EXPECT(zynum::const_matrix(m4, 3, 2, 2, &v) == Error::BufferTooSmall);
    EXPECT(zynum::const_matrix(m4, 4, -1, 2, &v) == Error::InvalidLength);
    double a6[6] = {1, 2, 3, 4, 5, 6}, b6[6] = {1, 2, 3, 4, 5, 6}, c4[4] = {0, 0, 0, 0};
    zynum::ConstMatrix<double> l, r;
    zynum::Matrix<double> out;
    EXPECT(zynum::const_matrix(a6, 6, 2, 3, &l) == Error::None);
    EXPECT(zynum::const_matrix(b6, 6, 2, 3, &r) == Error::None);
    EXPECT(zynum::matrix(c4, 4, 2, 2, &out) == Error::None);
    EXPECT(zynum::matrix_multiply(l, r, out) == Error::DimensionMismatch);
    // transposed right operand makes the shapes agree (no GPU work is done for the check itself)
    EXPECT(zynum::detail::check_shapes(l, r.transposed(), out) == Error::None);
    // zynum_test.zig:142-155: result aliasing an input
    double left[4] = {1, 2, 3, 4}, right[4] = {5, 6, 7, 8};
    EXPECT(zynum::const_matrix(left, 4, 2, 2, &l) == Error::None);
    EXPECT(zynum::const_matrix(right, 4, 2, 2, &r) == Error::None);
    EXPECT(zynum::matrix(left, 4, 2, 2, &out) == Error::None);
    EXPECT(zynum::matrix_multiply(l, r, out) == Error::AliasingNotAllowed);
    double ws[3];
    EXPECT(zynum::matrix_multiply_with_workspace(l, r, out, ws, 3) == Error::WorkspaceTooSmall);
    EXPECT(zynum::matrix_multiply_workspace_length(out) == 4);
}

static void compute() {
    // zynum_test.zig:28-41: 2x3 * 3x2
    double a[6] = {1, 2, 3, 4, 5, 6}, b[6] = {7, 8, 9, 10, 11, 12}, c[4] = {0, 0, 0, 0};
    zynum::ConstMatrix<double> l, r;
    zynum::Matrix<double> out;
    zynum::const_matrix(a, 6, 2, 3, &l);
    zynum::const_matrix(b, 6, 3, 2, &r);
    zynum::matrix(c, 4, 2, 2, &out);
    EXPECT(zynum::matrix_multiply(l, r, out) == Error::None);
    EXPECT(c[0] == 76 && c[1] == 100 && c[2] == 103 && c[3] == 136);
    // product_scale / result_scale and a transposed view
    double c2[4] = {1, 1, 1, 1};
    zynum::matrix(c2, 4, 2, 2, &out);
    zynum::ConstMatrix<double> at;
    zynum::const_matrix(a, 6, 3, 2, &at);  // the same storage seen as 3 x 2, used transposed
    EXPECT(zynum::matrix_multiply(at.transposed(), r, out, 2.0, -1.0) == Error::None);
    // at^T (2x3) = [[1,2,3],[4,5,6]]; times r = [[7,10],[8,11],[9,12]]
    EXPECT(c2[0] == 2 * 50 - 1 && c2[1] == 2 * 122 - 1 && c2[2] == 2 * 68 - 1 && c2[3] == 2 * 167 - 1);
    // zynum_test.zig:157-175: workspace form supports an in-place result
    double left[4] = {1, 2, 3, 4}, right[4] = {5, 6, 7, 8}, ws[4];
    zynum::const_matrix(left, 4, 2, 2, &l);
    zynum::const_matrix(right, 4, 2, 2, &r);
    zynum::matrix(left, 4, 2, 2, &out);
    EXPECT(zynum::matrix_multiply_with_workspace(l, r, out, ws, 4) == Error::None);
    EXPECT(left[0] == 23 && left[1] == 34 && left[2] == 31 && left[3] == 46);
    // complex
    std::complex<double> za[1] = {{2, 1}}, zb[1] = {{3, -1}}, zc[1] = {{0, 0}};
    zynum::ConstMatrix<std::complex<double>> zl, zr;
    zynum::Matrix<std::complex<double>> zo;
    zynum::const_matrix(za, 1, 1, 1, &zl);
    zynum::const_matrix(zb, 1, 1, 1, &zr);
    zynum::matrix(zc, 1, 1, 1, &zo);
    EXPECT(zynum::matrix_multiply(zl, zr, zo) == Error::None);
    EXPECT(zc[0] == std::complex<double>(7, 1));
}

int main(int argc, char** argv) {
    if (argc > 1 && !std::strcmp(argv[1], "compute"))
        compute();
    else
        checks();
    if (failures) return 1;
    std::printf("ok\n");
    return 0;
}
