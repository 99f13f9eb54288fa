// Explicitly rounded arithmetic.  The predictor must reproduce the reference
// build's rounding bit for bit, so every add/mul/fma below is an intrinsic the
// compiler may not re-contract or re-associate.  The contraction pattern is the
// one measured against the reference build on a B200: every expression was
// compared in all its fused variants and the matching one kept.
#pragma once
#include <cuda_runtime.h>

namespace prism_b200 {

template <class T> struct Fp;

template <> struct Fp<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ float abs(float a) { return fabsf(a); }
  static __device__ __forceinline__ int to_int_rz(float a) { return __float2int_rz(a); }
  static __device__ __forceinline__ float from_int(int a) { return __int2float_rn(a); }
  static __device__ __forceinline__ float from_double(double a) { return __double2float_rn(a); }
  // a value whose bits are the 32-bit word w (a code parked in a value slot)
  static __device__ __forceinline__ float with_low_word(int w) { return __int_as_float(w); }
};

template <> struct Fp<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
  static __device__ __forceinline__ double abs(double a) { return fabs(a); }
  static __device__ __forceinline__ int to_int_rz(double a) { return __double2int_rz(a); }
  static __device__ __forceinline__ double from_int(int a) { return __int2double_rn(a); }
  static __device__ __forceinline__ double from_double(double a) { return a; }
  // a value whose low word is w and whose high word is zero
  static __device__ __forceinline__ double with_low_word(int w) { return __hiloint2double(0, w); }
};

}  // namespace prism_b200
