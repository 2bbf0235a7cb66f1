// Complex scalars of the solve phase: cplx<float> (the complex64 factors of
// the mixed precision) and cplx<double> (complex128), laid out as {re, im}
// like std::complex and ParGeMSLR's ComplexValueClass (SRC/utils/complex.hpp),
// so interleaved host arrays map onto them directly.
//
// The kernels are templates over their value type; for a real T the helpers
// below reduce to the plain operation (conj(x) == x, abs2(x) == x * x), so the
// real instantiations perform exactly the arithmetic they did before complex
// types existed.
#pragma once

#include <cuda_runtime.h>

namespace pgx {

template <typename R>
struct __align__(2 * sizeof(R)) cplx {
  R x, y;
  cplx() = default;
  __host__ __device__ constexpr cplx(R re) : x(re), y(R(0)) {}
  __host__ __device__ constexpr cplx(R re, R im) : x(re), y(im) {}
  template <typename Q>
  __host__ __device__ explicit constexpr cplx(const cplx<Q>& o) : x(R(o.x)), y(R(o.y)) {}
  __host__ __device__ cplx& operator+=(const cplx& o) {
    x += o.x;
    y += o.y;
    return *this;
  }
  __host__ __device__ cplx& operator-=(const cplx& o) {
    x -= o.x;
    y -= o.y;
    return *this;
  }
  __host__ __device__ cplx& operator*=(const cplx& o) {
    const R re = x * o.x - y * o.y;
    y = x * o.y + y * o.x;
    x = re;
    return *this;
  }
};
template <typename R>
__host__ __device__ inline cplx<R> operator+(cplx<R> a, const cplx<R>& b) {
  return a += b;
}
template <typename R>
__host__ __device__ inline cplx<R> operator-(cplx<R> a, const cplx<R>& b) {
  return a -= b;
}
template <typename R>
__host__ __device__ inline cplx<R> operator-(const cplx<R>& a) {
  return cplx<R>(-a.x, -a.y);
}
template <typename R>
__host__ __device__ inline cplx<R> operator*(cplx<R> a, const cplx<R>& b) {
  return a *= b;
}
template <typename R>
__host__ __device__ inline cplx<R> operator*(const cplx<R>& a, R s) {
  return cplx<R>(a.x * s, a.y * s);
}
template <typename R>
__host__ __device__ inline cplx<R> operator*(R s, const cplx<R>& a) {
  return cplx<R>(a.x * s, a.y * s);
}
// a / b by the textbook formula a * conj(b) / |b|^2 (the reference's
// ComplexValueClass::operator/ divides the same way, SRC/utils/complex.hpp)
template <typename R>
__host__ __device__ inline cplx<R> operator/(const cplx<R>& a, const cplx<R>& b) {
  const R d = b.x * b.x + b.y * b.y;
  return cplx<R>((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
template <typename R>
__host__ __device__ inline cplx<R> operator/(const cplx<R>& a, R s) {
  return cplx<R>(a.x / s, a.y / s);
}
template <typename R>
__host__ __device__ inline bool operator==(const cplx<R>& a, const cplx<R>& b) {
  return a.x == b.x && a.y == b.y;
}

using cf32 = cplx<float>;
using cf64 = cplx<double>;

// scalar traits: the real type, complex-ness and the FP64 accumulator of T
template <typename T>
struct Sc {
  using real = T;
  using acc = double;  // reductions of the tall-skinny kernels
  static constexpr bool complex = false;
};
template <typename R>
struct Sc<cplx<R>> {
  using real = R;
  using acc = cf64;
  static constexpr bool complex = true;
};

__host__ __device__ inline float conj(float v) { return v; }
__host__ __device__ inline double conj(double v) { return v; }
template <typename R>
__host__ __device__ inline cplx<R> conj(const cplx<R>& v) {
  return cplx<R>(v.x, -v.y);
}
__host__ __device__ inline float abs2(float v) { return v * v; }
__host__ __device__ inline double abs2(double v) { return v * v; }
template <typename R>
__host__ __device__ inline R abs2(const cplx<R>& v) {
  return v.x * v.x + v.y * v.y;
}
// |v|: fabs for a real v; for a complex v sqrt(re^2 + im^2), as PargemslrAbs
__host__ __device__ inline double cabs(double v) { return fabs(v); }
__host__ __device__ inline float cabs(float v) { return fabsf(v); }
template <typename R>
__host__ __device__ inline R cabs(const cplx<R>& v) {
  return sqrt(v.x * v.x + v.y * v.y);
}
__host__ __device__ inline double re(double v) { return v; }
__host__ __device__ inline float re(float v) { return v; }
template <typename R>
__host__ __device__ inline R re(const cplx<R>& v) {
  return v.x;
}
__host__ __device__ inline bool finite_value(double v) { return isfinite(v); }
__host__ __device__ inline bool finite_value(float v) { return isfinite(v); }
template <typename R>
__host__ __device__ inline bool finite_value(const cplx<R>& v) {
  return isfinite(v.x) && isfinite(v.y);
}

// value conversion between the scalar types of one family (real to real,
// complex to complex, real to complex)
template <typename TO, typename TI>
__host__ __device__ inline TO to(const TI& v) {
  return TO(v);
}
template <>
__host__ __device__ inline cf32 to<cf32, cf64>(const cf64& v) {
  return cf32((float)v.x, (float)v.y);
}
template <>
__host__ __device__ inline cf64 to<cf64, cf32>(const cf32& v) {
  return cf64((double)v.x, (double)v.y);
}

// warp shuffles of a complex value: both parts
template <typename R>
__device__ inline cplx<R> __shfl_xor_sync(unsigned mask, const cplx<R>& v, int off) {
  return cplx<R>(::__shfl_xor_sync(mask, v.x, off), ::__shfl_xor_sync(mask, v.y, off));
}

}  // namespace pgx
