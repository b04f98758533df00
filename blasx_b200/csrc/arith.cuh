// arith.cuh -- element arithmetic shared by the SIMT kernels: real float /
// double and interleaved complex pairs (complex64 c2, complex128 z2), with
// the host-side conversion of a (re, im) scalar.
#pragma once

#include "runtime.h"

namespace bx {

struct z2 {
    double re, im;
};
struct c2 {  // complex64: interleaved (re, im) floats
    float re, im;
};

template <typename T> struct Arith;

template <> struct Arith<float> {
    using V = float;
    __device__ static V zero() { return 0.f; }
    __device__ static V one() { return 1.f; }
    __device__ static V real_part(V a) { return a; }
    __device__ static V fma(V a, V b, V c) { return fmaf(a, b, c); }
    __device__ static V conj(V a) { return a; }
    __device__ static V mul(V a, V b) { return a * b; }
    __device__ static V add(V a, V b) { return a + b; }
};
template <> struct Arith<double> {
    using V = double;
    __device__ static V zero() { return 0.0; }
    __device__ static V one() { return 1.0; }
    __device__ static V real_part(V a) { return a; }
    __device__ static V fma(V a, V b, V c) { return ::fma(a, b, c); }
    __device__ static V conj(V a) { return a; }
    __device__ static V mul(V a, V b) { return a * b; }
    __device__ static V add(V a, V b) { return a + b; }
};
template <> struct Arith<z2> {
    using V = z2;
    __device__ static V zero() { return {0.0, 0.0}; }
    __device__ static V one() { return {1.0, 0.0}; }
    __device__ static V real_part(V a) { return {a.re, 0.0}; }
    __device__ static V fma(V a, V b, V c) {
        c.re = ::fma(a.re, b.re, c.re);
        c.re = ::fma(-a.im, b.im, c.re);
        c.im = ::fma(a.re, b.im, c.im);
        c.im = ::fma(a.im, b.re, c.im);
        return c;
    }
    __device__ static V conj(V a) { return {a.re, -a.im}; }
    __device__ static V mul(V a, V b) {
        return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    }
    __device__ static V add(V a, V b) { return {a.re + b.re, a.im + b.im}; }
};

template <> struct Arith<c2> {
    using V = c2;
    __device__ static V zero() { return {0.f, 0.f}; }
    __device__ static V one() { return {1.f, 0.f}; }
    __device__ static V real_part(V a) { return {a.re, 0.f}; }
    __device__ static V fma(V a, V b, V c) {
        c.re = fmaf(a.re, b.re, c.re);
        c.re = fmaf(-a.im, b.im, c.re);
        c.im = fmaf(a.re, b.im, c.im);
        c.im = fmaf(a.im, b.re, c.im);
        return c;
    }
    __device__ static V conj(V a) { return {a.re, -a.im}; }
    __device__ static V mul(V a, V b) {
        return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    }
    __device__ static V add(V a, V b) { return {a.re + b.re, a.im + b.im}; }
};

template <typename T> __host__ T from_cplx(cplx c);
template <> inline __host__ float from_cplx<float>(cplx c) { return float(c.re); }
template <> inline __host__ double from_cplx<double>(cplx c) { return c.re; }
template <> inline __host__ z2 from_cplx<z2>(cplx c) { return {c.re, c.im}; }
template <> inline __host__ c2 from_cplx<c2>(cplx c) { return {float(c.re), float(c.im)}; }

// Quotient a / b. Complex: Smith's algorithm (scaling by the larger part of
// b), which avoids the overflow and underflow of the textbook formula.
template <typename T> __device__ inline T quot(T a, T b) { return a / b; }
template <> __device__ inline z2 quot<z2>(z2 a, z2 b) {
    if (fabs(b.re) >= fabs(b.im)) {
        const double r = b.im / b.re, d = b.re + b.im * r;
        return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
    }
    const double r = b.re / b.im, d = b.im + b.re * r;
    return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
template <> __device__ inline c2 quot<c2>(c2 a, c2 b) {
    if (fabsf(b.re) >= fabsf(b.im)) {
        const float r = b.im / b.re, d = b.re + b.im * r;
        return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
    }
    const float r = b.re / b.im, d = b.im + b.re * r;
    return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}

}  // namespace bx
