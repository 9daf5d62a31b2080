// Shim for the reference's external qcu_io header base/datatype/qcu_complex.cuh:
// a complex number with the storage layout of Float2_t<T> (the kernels reinterpret
// arrays of one as the other) and textbook arithmetic.
#pragma once
#include "base/datatype/qcu_float2.cuh"

template <typename T>
struct Complex {
    T re, im;
    __host__ __device__ Complex() : re(0), im(0) {}
    __host__ __device__ Complex(T r, T i) : re(r), im(i) {}
    __host__ __device__ Complex(int r) : re(T(r)), im(0) {}
    __host__ __device__ Complex(const qcu::Float2_t<T>& v) : re(v.x), im(v.y) {}
    __host__ __device__ T real() const { return re; }
    __host__ __device__ T imag() const { return im; }
    __host__ __device__ Complex conj() const { return Complex(re, -im); }
    __host__ __device__ T norm2() const { return re * re + im * im; }
    __host__ __device__ Complex operator-() const { return Complex(-re, -im); }
    __host__ __device__ Complex operator+(const Complex& o) const { return Complex(re + o.re, im + o.im); }
    __host__ __device__ Complex operator-(const Complex& o) const { return Complex(re - o.re, im - o.im); }
    __host__ __device__ Complex operator*(const Complex& o) const {
        return Complex(re * o.re - im * o.im, re * o.im + im * o.re);
    }
    __host__ __device__ Complex operator*(T s) const { return Complex(re * s, im * s); }
    __host__ __device__ Complex& operator+=(const Complex& o) {
        re += o.re;
        im += o.im;
        return *this;
    }
    __host__ __device__ Complex& operator=(int v) {
        re = T(v);
        im = 0;
        return *this;
    }
    __host__ __device__ operator qcu::Float2_t<T>() const {
        qcu::Float2_t<T> v;
        v.x = re;
        v.y = im;
        return v;
    }
};
