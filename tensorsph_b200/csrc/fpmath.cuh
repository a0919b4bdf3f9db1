// IEEE round-to-nearest arithmetic with no contraction, per dtype.
//
// The reference evaluates every elementwise op as a separately rounded
// PyTorch kernel; where integer results (cell keys, pair membership) depend on
// the last bit, the CUDA path uses the same rounded operations.
#pragma once

#include <cuda_runtime.h>

namespace tsph {

template <class T>
struct fp;

template <>
struct fp<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
  // delta - box * round_half_even(delta / box)  (threed/neighbors3.py:45-53)
  static __device__ __forceinline__ float min_image(float d, float box) {
    return sub(d, mul(box, rintf(div(d, box))));
  }
};

template <>
struct fp<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
  static __device__ __forceinline__ double min_image(double d, double box) {
    return sub(d, mul(box, rint(div(d, box))));
  }
};

}  // namespace tsph
