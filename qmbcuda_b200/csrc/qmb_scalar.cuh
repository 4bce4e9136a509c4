// qmb_scalar.cuh -- real / complex scalar helpers in FP32 and FP64.
#pragma once
#include <cuda_runtime.h>

namespace qmb {

template <class T> struct Sc;

template <> struct Sc<double> {
    using real = double;
    static constexpr bool cplx = false;
    __host__ __device__ static double zero() { return 0.0; }
    __host__ __device__ static double from(double2 v) { return v.x; }
    __host__ __device__ static double2 to2(double v) { return make_double2(v, 0.0); }
    __host__ __device__ static double mul(double a, double b) { return a * b; }
    __host__ __device__ static double add(double a, double b) { return a + b; }
    __host__ __device__ static double sub(double a, double b) { return a - b; }
    __host__ __device__ static double scale(double a, double s) { return a * s; }
    __host__ __device__ static double fma(double a, double b, double c) { return ::fma(a, b, c); }
    __host__ __device__ static double re_conj_mul(double a, double b) { return a * b; }
    __host__ __device__ static double im_conj_mul(double, double) { return 0.0; }
    __host__ __device__ static double abs2(double a) { return a * a; }
};

template <> struct Sc<float> {
    using real = float;
    static constexpr bool cplx = false;
    __host__ __device__ static float zero() { return 0.0f; }
    __host__ __device__ static float from(double2 v) { return (float)v.x; }
    __host__ __device__ static double2 to2(float v) { return make_double2(v, 0.0); }
    __host__ __device__ static float mul(float a, float b) { return a * b; }
    __host__ __device__ static float add(float a, float b) { return a + b; }
    __host__ __device__ static float sub(float a, float b) { return a - b; }
    __host__ __device__ static float scale(float a, double s) { return (float)(a * s); }
    // a float factor: the product of two floats is exact in double, so the
    // rounded float product equals the double form above
    __host__ __device__ static float scale(float a, float s) { return a * s; }
    __host__ __device__ static float fma(float a, float b, float c) { return fmaf(a, b, c); }
    __host__ __device__ static double re_conj_mul(float a, float b) { return (double)a * b; }
    __host__ __device__ static double im_conj_mul(float, float) { return 0.0; }
    __host__ __device__ static double abs2(float a) { return (double)a * a; }
};

template <> struct Sc<double2> {
    using real = double;
    static constexpr bool cplx = true;
    __host__ __device__ static double2 zero() { return make_double2(0.0, 0.0); }
    __host__ __device__ static double2 from(double2 v) { return v; }
    __host__ __device__ static double2 to2(double2 v) { return v; }
    __host__ __device__ static double2 mul(double2 a, double2 b) {
        return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    }
    __host__ __device__ static double2 add(double2 a, double2 b) {
        return make_double2(a.x + b.x, a.y + b.y);
    }
    __host__ __device__ static double2 sub(double2 a, double2 b) {
        return make_double2(a.x - b.x, a.y - b.y);
    }
    __host__ __device__ static double2 scale(double2 a, double s) {
        return make_double2(a.x * s, a.y * s);
    }
    __host__ __device__ static double2 fma(double2 a, double2 b, double2 c) {
        return make_double2(::fma(a.x, b.x, ::fma(-a.y, b.y, c.x)),
                            ::fma(a.x, b.y, ::fma(a.y, b.x, c.y)));
    }
    __host__ __device__ static double re_conj_mul(double2 a, double2 b) {
        return a.x * b.x + a.y * b.y;
    }
    __host__ __device__ static double im_conj_mul(double2 a, double2 b) {
        return a.x * b.y - a.y * b.x;
    }
    __host__ __device__ static double abs2(double2 a) { return a.x * a.x + a.y * a.y; }
};

template <> struct Sc<float2> {
    using real = float;
    static constexpr bool cplx = true;
    __host__ __device__ static float2 zero() { return make_float2(0.0f, 0.0f); }
    __host__ __device__ static float2 from(double2 v) { return make_float2((float)v.x, (float)v.y); }
    __host__ __device__ static double2 to2(float2 v) { return make_double2(v.x, v.y); }
    __host__ __device__ static float2 mul(float2 a, float2 b) {
        return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    }
    __host__ __device__ static float2 add(float2 a, float2 b) {
        return make_float2(a.x + b.x, a.y + b.y);
    }
    __host__ __device__ static float2 sub(float2 a, float2 b) {
        return make_float2(a.x - b.x, a.y - b.y);
    }
    __host__ __device__ static float2 scale(float2 a, double s) {
        return make_float2((float)(a.x * s), (float)(a.y * s));
    }
    // a float factor: same rounding as the double form (exact double product)
    __host__ __device__ static float2 scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
    __host__ __device__ static float2 fma(float2 a, float2 b, float2 c) {
        return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
    }
    __host__ __device__ static double re_conj_mul(float2 a, float2 b) {
        return (double)a.x * b.x + (double)a.y * b.y;
    }
    __host__ __device__ static double im_conj_mul(float2 a, float2 b) {
        return (double)a.x * b.y - (double)a.y * b.x;
    }
    __host__ __device__ static double abs2(float2 a) { return (double)a.x * a.x + (double)a.y * a.y; }
};

// conversion between vector scalar types of the same kind
template <class To, class From> __host__ __device__ inline To cvt(From v);
template <> __host__ __device__ inline double cvt<double, double>(double v) { return v; }
template <> __host__ __device__ inline float cvt<float, float>(float v) { return v; }
template <> __host__ __device__ inline double cvt<double, float>(float v) { return v; }
template <> __host__ __device__ inline float cvt<float, double>(double v) { return (float)v; }
template <> __host__ __device__ inline double2 cvt<double2, double2>(double2 v) { return v; }
template <> __host__ __device__ inline float2 cvt<float2, float2>(float2 v) { return v; }
template <> __host__ __device__ inline double2 cvt<double2, float2>(float2 v) {
    return make_double2(v.x, v.y);
}
template <> __host__ __device__ inline float2 cvt<float2, double2>(double2 v) {
    return make_float2((float)v.x, (float)v.y);
}

}  // namespace qmb
