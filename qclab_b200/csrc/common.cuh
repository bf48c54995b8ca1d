// Device-side element types and exact (non-contracted) complex arithmetic.
//
// The reference multiplies std::complex values as (ac - bd, ad + bc) and
// adds component-wise, each step rounded (g++ on x86-64 without FMA).
// The *_rn intrinsics keep every product and sum separately rounded so the
// reference-exact kernels reproduce those values bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qsv {

// ---- element traits -------------------------------------------------------
template <typename V> struct Elem;
template <> struct Elem<double2> { using R = double; static constexpr bool cplx = true;  };
template <> struct Elem<float2>  { using R = float;  static constexpr bool cplx = true;  };
template <> struct Elem<double>  { using R = double; static constexpr bool cplx = false; };
template <> struct Elem<float>   { using R = float;  static constexpr bool cplx = false; };

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float  mul_rn(float a, float b)   { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float  add_rn(float a, float b)   { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float  sub_rn(float a, float b)   { return __fsub_rn(a, b); }

// m * x, exactly as std::complex operator* evaluates it.
__device__ __forceinline__ double2 emul(double2 m, double2 x) {
  return make_double2(sub_rn(mul_rn(m.x, x.x), mul_rn(m.y, x.y)),
                      add_rn(mul_rn(m.x, x.y), mul_rn(m.y, x.x)));
}
__device__ __forceinline__ float2 emul(float2 m, float2 x) {
  return make_float2(sub_rn(mul_rn(m.x, x.x), mul_rn(m.y, x.y)),
                     add_rn(mul_rn(m.x, x.y), mul_rn(m.y, x.x)));
}
__device__ __forceinline__ double emul(double m, double x) { return mul_rn(m, x); }
__device__ __forceinline__ float  emul(float m, float x)   { return mul_rn(m, x); }

__device__ __forceinline__ double2 eadd(double2 a, double2 b) {
  return make_double2(add_rn(a.x, b.x), add_rn(a.y, b.y));
}
__device__ __forceinline__ float2 eadd(float2 a, float2 b) {
  return make_float2(add_rn(a.x, b.x), add_rn(a.y, b.y));
}
__device__ __forceinline__ double eadd(double a, double b) { return add_rn(a, b); }
__device__ __forceinline__ float  eadd(float a, float b)   { return add_rn(a, b); }

__device__ __forceinline__ double2 esub(double2 a, double2 b) {
  return make_double2(sub_rn(a.x, b.x), sub_rn(a.y, b.y));
}
__device__ __forceinline__ float2 esub(float2 a, float2 b) {
  return make_float2(sub_rn(a.x, b.x), sub_rn(a.y, b.y));
}
__device__ __forceinline__ double esub(double a, double b) { return sub_rn(a, b); }
__device__ __forceinline__ float  esub(float a, float b)   { return sub_rn(a, b); }

// s * x for a real scalar s (std::complex's real-scalar operator*: each
// component times s)
__device__ __forceinline__ double2 smul(double s, double2 x) {
  return make_double2(mul_rn(s, x.x), mul_rn(s, x.y));
}
__device__ __forceinline__ float2 smul(float s, float2 x) {
  return make_float2(mul_rn(s, x.x), mul_rn(s, x.y));
}
__device__ __forceinline__ double smul(double s, double x) { return mul_rn(s, x); }
__device__ __forceinline__ float  smul(float s, float x)   { return mul_rn(s, x); }

// -x (std::complex's unary minus: each component negated)
__device__ __forceinline__ double2 eneg(double2 x) { return make_double2(-x.x, -x.y); }
__device__ __forceinline__ float2  eneg(float2 x)  { return make_float2(-x.x, -x.y); }
__device__ __forceinline__ double  eneg(double x)  { return -x; }
__device__ __forceinline__ float   eneg(float x)   { return -x; }

// real part of a coefficient
__device__ __forceinline__ double ere(double2 m) { return m.x; }
__device__ __forceinline__ float  ere(float2 m)  { return m.x; }
__device__ __forceinline__ double ere(double m)  { return m; }
__device__ __forceinline__ float  ere(float m)   { return m; }

// ---- fast (FMA-contracted) arithmetic for the fused sweeps ----------------
__device__ __forceinline__ double2 fmul(double2 m, double2 x) {
  return make_double2(fma(m.x, x.x, -m.y * x.y), fma(m.x, x.y, m.y * x.x));
}
__device__ __forceinline__ float2 fmul(float2 m, float2 x) {
  return make_float2(fmaf(m.x, x.x, -m.y * x.y), fmaf(m.x, x.y, m.y * x.x));
}
// acc + m * x
__device__ __forceinline__ double2 fmac(double2 acc, double2 m, double2 x) {
  return make_double2(fma(-m.y, x.y, fma(m.x, x.x, acc.x)),
                      fma(m.y, x.x, fma(m.x, x.y, acc.y)));
}
__device__ __forceinline__ float2 fmac(float2 acc, float2 m, float2 x) {
  return make_float2(fmaf(-m.y, x.y, fmaf(m.x, x.x, acc.x)),
                     fmaf(m.y, x.x, fmaf(m.x, x.y, acc.y)));
}

template <typename V> __device__ __forceinline__ V vzero();
template <> __device__ __forceinline__ double2 vzero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2  vzero<float2>()  { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double  vzero<double>()  { return 0.0; }
template <> __device__ __forceinline__ float   vzero<float>()   { return 0.f; }

// Coefficient (matrix entry) of the same kind as the element.
template <typename V> struct Coef { using type = V; };

template <typename V> __device__ __forceinline__ V coef(const double* m, int i);
template <> __device__ __forceinline__ double2 coef<double2>(const double* m, int i) {
  return make_double2(m[2 * i], m[2 * i + 1]);
}
template <> __device__ __forceinline__ float2 coef<float2>(const double* m, int i) {
  return make_float2((float)m[2 * i], (float)m[2 * i + 1]);
}
template <> __device__ __forceinline__ double coef<double>(const double* m, int i) {
  return m[2 * i];
}
template <> __device__ __forceinline__ float coef<float>(const double* m, int i) {
  return (float)m[2 * i];
}

__device__ __forceinline__ double2 shfl_xor(double2 v, int mask) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, mask),
                      __shfl_xor_sync(0xffffffffu, v.y, mask));
}
__device__ __forceinline__ float2 shfl_xor(float2 v, int mask) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, mask),
                     __shfl_xor_sync(0xffffffffu, v.y, mask));
}
__device__ __forceinline__ double shfl_xor(double v, int mask) {
  return __shfl_xor_sync(0xffffffffu, v, mask);
}
__device__ __forceinline__ float shfl_xor(float v, int mask) {
  return __shfl_xor_sync(0xffffffffu, v, mask);
}
__device__ __forceinline__ double2 shfl_idx(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src),
                      __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ float2 shfl_idx(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src),
                     __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ double shfl_idx(double v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}
__device__ __forceinline__ float shfl_idx(float v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}

// Inserts a zero bit at position p of x.
__host__ __device__ __forceinline__ uint64_t insert_zero(uint64_t x, int p) {
  const uint64_t lo = x & ((1ull << p) - 1ull);
  return ((x >> p) << (p + 1)) | lo;
}

}  // namespace qsv
