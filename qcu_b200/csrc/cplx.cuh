// Small complex type used by every kernel.  T is the arithmetic type (double
// for the FP64 path, float for the FP32 and FP16-storage paths).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace qcu {

template <typename T>
struct Cpx {
  T re, im;
  __host__ __device__ __forceinline__ Cpx() {}
  __host__ __device__ __forceinline__ constexpr Cpx(T r, T i) : re(r), im(i) {}
  __host__ __device__ __forceinline__ Cpx operator+(const Cpx &o) const { return {re + o.re, im + o.im}; }
  __host__ __device__ __forceinline__ Cpx operator-(const Cpx &o) const { return {re - o.re, im - o.im}; }
  __host__ __device__ __forceinline__ Cpx operator-() const { return {-re, -im}; }
  __host__ __device__ __forceinline__ Cpx operator*(const Cpx &o) const {
    return {re * o.re - im * o.im, re * o.im + im * o.re};
  }
  __host__ __device__ __forceinline__ Cpx operator*(T s) const { return {re * s, im * s}; }
  __host__ __device__ __forceinline__ Cpx &operator+=(const Cpx &o) {
    re += o.re;
    im += o.im;
    return *this;
  }
  __host__ __device__ __forceinline__ Cpx &operator-=(const Cpx &o) {
    re -= o.re;
    im -= o.im;
    return *this;
  }
  __host__ __device__ __forceinline__ Cpx conj() const { return {re, -im}; }
  __host__ __device__ __forceinline__ T norm2() const { return re * re + im * im; }
};

template <typename T>
__host__ __device__ __forceinline__ Cpx<T> cmake(T r, T i) {
  return Cpx<T>(r, i);
}

// conj(a) * b
template <typename T>
__host__ __device__ __forceinline__ Cpx<T> cdotmul(const Cpx<T> &a, const Cpx<T> &b) {
  return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}

// multiply by a unit constant (re,im) in {(1,0),(-1,0),(0,1),(0,-1)}, folded at compile time
template <int RE, int IM, typename T>
__host__ __device__ __forceinline__ Cpx<T> unit_mul(const Cpx<T> &z) {
  static_assert(RE * RE + IM * IM == 1, "unit constant");
  if constexpr (RE == 1) return z;
  else if constexpr (RE == -1) return -z;
  else if constexpr (IM == 1) return {-z.im, z.re};
  else return {z.im, -z.re};
}

// complex division a / b
template <typename T>
__host__ __device__ __forceinline__ Cpx<T> cdiv(const Cpx<T> &a, const Cpx<T> &b) {
  T d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}

}  // namespace qcu
