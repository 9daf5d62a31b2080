// Shim for the reference's external qcu_io header base/datatype/qcu_float2.cuh:
// the complex storage pair of a real type (double2, float2, half2).
#pragma once
#include <cuda_fp16.h>

namespace qcu {
template <typename T> struct Float2Wrapper;
template <> struct Float2Wrapper<double> { using Float = double; using Float2 = double2; };
template <> struct Float2Wrapper<float> { using Float = float; using Float2 = float2; };
template <> struct Float2Wrapper<half> { using Float = half; using Float2 = half2; };
template <typename T> using Float2_t = typename Float2Wrapper<T>::Float2;
}  // namespace qcu
using qcu::Float2_t;
