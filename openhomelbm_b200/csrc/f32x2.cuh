// Packed binary32 pair arithmetic for sm_100a (FADD2 / FMUL2 / FFMA2).
//
// P2 holds the same quantity for two cells; every operator issues ONE packed instruction
// for both. A product is kept pending (M2) so that `a * b + c` becomes one fused
// multiply-add, as the compiler would contract it for scalars. Each lane rounds exactly as
// the scalar operation would (round to nearest even). Division is lane-wise.
#pragma once

#include <cuda_runtime.h>

namespace hl {

struct M2;

struct P2 {
  float2 v;
  P2() = default;
  __device__ __forceinline__ explicit P2(float2 a) : v(a) {}
  __device__ __forceinline__ P2(float a, float b) : v(make_float2(a, b)) {}
  // broadcast constant (the scalar code's R(c))
  __device__ __forceinline__ P2(double c) : v(make_float2(float(c), float(c))) {}
  __device__ __forceinline__ P2(const M2& m);
  __device__ __forceinline__ float x() const { return v.x; }
  __device__ __forceinline__ float y() const { return v.y; }
};

// pending product a * b
struct M2 {
  float2 a, b;
};

__device__ __forceinline__ P2::P2(const M2& m) : v(__fmul2_rn(m.a, m.b)) {}

__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

__device__ __forceinline__ P2 operator+(P2 a, P2 b) { return P2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ P2 operator-(P2 a, P2 b) { return P2(__fadd2_rn(a.v, neg2(b.v))); }
__device__ __forceinline__ P2 operator-(P2 a) { return P2(neg2(a.v)); }
__device__ __forceinline__ M2 operator*(P2 a, P2 b) { return M2{a.v, b.v}; }
__device__ __forceinline__ M2 operator*(const M2& m, P2 b) { return M2{__fmul2_rn(m.a, m.b), b.v}; }
__device__ __forceinline__ M2 operator*(P2 a, const M2& m) { return M2{a.v, __fmul2_rn(m.a, m.b)}; }
__device__ __forceinline__ M2 operator*(const M2& m, const M2& n) { return M2{__fmul2_rn(m.a, m.b), __fmul2_rn(n.a, n.b)}; }
__device__ __forceinline__ M2 operator-(const M2& m) { return M2{neg2(m.a), m.b}; }
__device__ __forceinline__ P2 operator+(const M2& m, P2 c) { return P2(__ffma2_rn(m.a, m.b, c.v)); }
__device__ __forceinline__ P2 operator+(P2 c, const M2& m) { return P2(__ffma2_rn(m.a, m.b, c.v)); }
__device__ __forceinline__ P2 operator-(const M2& m, P2 c) { return P2(__ffma2_rn(m.a, m.b, neg2(c.v))); }
__device__ __forceinline__ P2 operator-(P2 c, const M2& m) { return P2(__ffma2_rn(neg2(m.a), m.b, c.v)); }
__device__ __forceinline__ P2 operator+(const M2& m, const M2& n) { return P2(__ffma2_rn(m.a, m.b, __fmul2_rn(n.a, n.b))); }
__device__ __forceinline__ P2 operator-(const M2& m, const M2& n) {
  return P2(__ffma2_rn(m.a, m.b, neg2(__fmul2_rn(n.a, n.b))));
}
__device__ __forceinline__ P2 operator/(P2 a, P2 b) { return P2(a.v.x / b.v.x, a.v.y / b.v.y); }
__device__ __forceinline__ P2& operator+=(P2& a, P2 b) { return a = a + b; }
__device__ __forceinline__ P2& operator-=(P2& a, P2 b) { return a = a - b; }
__device__ __forceinline__ P2& operator+=(P2& a, const M2& m) { return a = a + m; }
__device__ __forceinline__ P2 fmax(P2 a, P2 b) { return P2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y)); }
// {a.y, b.x}: the lanes that straddle two consecutive pairs
__device__ __forceinline__ P2 funnel(P2 a, P2 b) { return P2(a.v.y, b.v.x); }

}  // namespace hl
