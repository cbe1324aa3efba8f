// Small elementwise kernels shared by every GEMM-family entry point.
#include "common.cuh"
#include "kernels.h"

namespace zb {
namespace {

template <typename T>
__global__ void scale_matrix_kernel(int m, int n, T beta, T* __restrict__ c, long ldc) {
    long total = (long)m * n;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        int i = (int)(q % m), j = (int)(q / m);
        T* p = c + (long)j * ldc + i;
        *p = (beta == T(0)) ? T(0) : beta * *p;
    }
}

template <typename T>
__global__ void scale_matrix_complex_kernel(int m, int n, T br, T bi, T* __restrict__ c, long ldc) {
    long total = (long)m * n;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        int i = (int)(q % m), j = (int)(q / m);
        T* p = c + 2 * ((long)j * ldc + i);
        if (br == T(0) && bi == T(0)) {
            p[0] = T(0);
            p[1] = T(0);
        } else {
            T r = br * p[0] - bi * p[1], s = br * p[1] + bi * p[0];
            p[0] = r;
            p[1] = s;
        }
    }
}

inline int grid_for(long total) {
    long b = (total + 255) / 256;
    if (b > 148L * 32) b = 148L * 32;
    return b < 1 ? 1 : (int)b;
}

}  // namespace

cudaError_t scale_matrix_f64(int m, int n, double beta, double* c, long ldc, cudaStream_t st) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    scale_matrix_kernel<double><<<grid_for((long)m * n), 256, 0, st>>>(m, n, beta, c, ldc);
    count_launch();
    return cudaGetLastError();
}
cudaError_t scale_matrix_f32(int m, int n, float beta, float* c, long ldc, cudaStream_t st) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    scale_matrix_kernel<float><<<grid_for((long)m * n), 256, 0, st>>>(m, n, beta, c, ldc);
    count_launch();
    return cudaGetLastError();
}
cudaError_t scale_matrix_z(int m, int n, const double* beta, double* c, long ldc, cudaStream_t st) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    scale_matrix_complex_kernel<double><<<grid_for((long)m * n), 256, 0, st>>>(m, n, beta[0], beta[1], c, ldc);
    count_launch();
    return cudaGetLastError();
}
cudaError_t scale_matrix_c(int m, int n, const float* beta, float* c, long ldc, cudaStream_t st) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    scale_matrix_complex_kernel<float><<<grid_for((long)m * n), 256, 0, st>>>(m, n, beta[0], beta[1], c, ldc);
    count_launch();
    return cudaGetLastError();
}

}  // namespace zb
