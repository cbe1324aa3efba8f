// Interleaved complex number (re, im) for the complex TRSM / SYRK paths: the
// same memory layout as the reference's ComplexF64 / ComplexF32 extern structs
// (types.zig), with the reference's scalar arithmetic (core/shared/scalar.zig:
// mul :77 (a.re b.re - a.im b.im, a.re b.im + a.im b.re), divv :84, conj :92).
// Overloads of fma / shuffles / conj_if let the generic TRSM kernels run on
// real and complex element types alike.
#pragma once

#include <cuda_runtime.h>

namespace zb {

#ifdef __CUDACC__
// the overloads below would hide the global real ones inside namespace zb
using ::fma;
using ::__shfl_sync;
using ::__shfl_xor_sync;
#endif

template <typename R>
struct cnum {
    R re, im;
    cnum() = default;
    __host__ __device__ constexpr cnum(R r, R i = R(0)) : re(r), im(i) {}
};

template <typename R>
__host__ __device__ inline cnum<R> operator+(cnum<R> a, cnum<R> b) {
    return {a.re + b.re, a.im + b.im};
}
template <typename R>
__host__ __device__ inline cnum<R> operator-(cnum<R> a, cnum<R> b) {
    return {a.re - b.re, a.im - b.im};
}
template <typename R>
__host__ __device__ inline cnum<R> operator-(cnum<R> a) {
    return {-a.re, -a.im};
}
template <typename R>
__host__ __device__ inline cnum<R> operator*(cnum<R> a, cnum<R> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R>
__host__ __device__ inline cnum<R> operator/(cnum<R> a, cnum<R> b) {
    const R den = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den};
}
template <typename R>
__host__ __device__ inline cnum<R>& operator+=(cnum<R>& a, cnum<R> b) {
    a.re += b.re;
    a.im += b.im;
    return a;
}
template <typename R>
__host__ __device__ inline cnum<R>& operator-=(cnum<R>& a, cnum<R> b) {
    a.re -= b.re;
    a.im -= b.im;
    return a;
}
template <typename R>
__host__ __device__ inline bool operator==(cnum<R> a, cnum<R> b) {
    return a.re == b.re && a.im == b.im;
}
template <typename R>
__host__ __device__ inline bool operator!=(cnum<R> a, cnum<R> b) {
    return !(a == b);
}

#ifdef __CUDACC__
// a * b + c
template <typename R>
__device__ inline cnum<R> fma(cnum<R> a, cnum<R> b, cnum<R> c) {
    return {::fma(a.re, b.re, ::fma(-a.im, b.im, c.re)), ::fma(a.re, b.im, ::fma(a.im, b.re, c.im))};
}

template <typename R>
__device__ inline cnum<R> __shfl_sync(unsigned mask, cnum<R> v, int src) {
    return {::__shfl_sync(mask, v.re, src), ::__shfl_sync(mask, v.im, src)};
}
template <typename R>
__device__ inline cnum<R> __shfl_xor_sync(unsigned mask, cnum<R> v, int lane_mask) {
    return {::__shfl_xor_sync(mask, v.re, lane_mask), ::__shfl_xor_sync(mask, v.im, lane_mask)};
}
#endif

// conj(v) when c (complex), v unchanged (real)
__host__ __device__ inline double conj_if(double v, bool) { return v; }
__host__ __device__ inline float conj_if(float v, bool) { return v; }
template <typename R>
__host__ __device__ inline cnum<R> conj_if(cnum<R> v, bool c) {
    return c ? cnum<R>{v.re, -v.im} : v;
}

// a Hermitian matrix's diagonal: the real part only (when h, complex), v unchanged otherwise
__host__ __device__ inline double herm_diag(double v, bool) { return v; }
__host__ __device__ inline float herm_diag(float v, bool) { return v; }
template <typename R>
__host__ __device__ inline cnum<R> herm_diag(cnum<R> v, bool h) {
    return h ? cnum<R>{v.re, R(0)} : v;
}

template <typename T>
struct is_cnum {
    static constexpr bool value = false;
};
template <typename R>
struct is_cnum<cnum<R>> {
    static constexpr bool value = true;
};

}  // namespace zb
