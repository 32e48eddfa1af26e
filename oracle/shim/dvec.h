/*
 * Project-written stand-in for the Intel compiler's <dvec.h>, used ONLY to
 * compile the reference CPU solver (scalar/src/cpu/trid_cpu.cpp) with g++
 * as the test oracle / CPU baseline.  Test infrastructure, never shipped.
 *
 * trid_cpu.cpp (through include/trid_simd.h) needs:
 *   - F64vec4 / F32vec8: a 32-byte SIMD value type with + - * / and +=,
 *     constructible from a scalar and convertible to/from __m256d / __m256;
 *   - __assume_aligned(ptr, n): an Intel alignment hint (a no-op here).
 */
#ifndef ORACLE_DVEC_SHIM_H
#define ORACLE_DVEC_SHIM_H

#include <immintrin.h>

#define __assume_aligned(ptr, n) ((void)0)

struct F64vec4 {
  __m256d v;
  F64vec4() {}
  F64vec4(__m256d x) : v(x) {}
  explicit F64vec4(double s) : v(_mm256_set1_pd(s)) {}
  operator __m256d() const { return v; }
  F64vec4 &operator+=(const F64vec4 &o) { v = _mm256_add_pd(v, o.v); return *this; }
};
inline F64vec4 operator+(const F64vec4 &x, const F64vec4 &y) { return _mm256_add_pd(x.v, y.v); }
inline F64vec4 operator-(const F64vec4 &x, const F64vec4 &y) { return _mm256_sub_pd(x.v, y.v); }
inline F64vec4 operator*(const F64vec4 &x, const F64vec4 &y) { return _mm256_mul_pd(x.v, y.v); }
inline F64vec4 operator/(const F64vec4 &x, const F64vec4 &y) { return _mm256_div_pd(x.v, y.v); }

struct F32vec8 {
  __m256 v;
  F32vec8() {}
  F32vec8(__m256 x) : v(x) {}
  explicit F32vec8(float s) : v(_mm256_set1_ps(s)) {}
  operator __m256() const { return v; }
  F32vec8 &operator+=(const F32vec8 &o) { v = _mm256_add_ps(v, o.v); return *this; }
};
inline F32vec8 operator+(const F32vec8 &x, const F32vec8 &y) { return _mm256_add_ps(x.v, y.v); }
inline F32vec8 operator-(const F32vec8 &x, const F32vec8 &y) { return _mm256_sub_ps(x.v, y.v); }
inline F32vec8 operator*(const F32vec8 &x, const F32vec8 &y) { return _mm256_mul_ps(x.v, y.v); }
inline F32vec8 operator/(const F32vec8 &x, const F32vec8 &y) { return _mm256_div_ps(x.v, y.v); }

#endif
