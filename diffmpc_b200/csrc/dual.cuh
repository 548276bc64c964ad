// Forward-mode dual and hyper-dual numbers for device code.
//
// Dual  = v + d e            (e^2 = 0): one Jacobian column per evaluation; this
//         replaces the reference's `value_and_jacfwd` (diffmpc/utils/jax_utils.py:12-36).
// HDual = v + a e1 + b e2 + ab e1e2 (e1^2 = e2^2 = 0): the e1e2 part of f(z + z~ e1,
//         theta + e2) is the mixed second derivative (d^2 f / dz dtheta) . z~, which
//         replaces the reference's nested jacfwd over weights (sqp.py:620-641).
#pragma once
#include <cuda_runtime.h>

struct Dual {
  double v, d;
  __device__ __forceinline__ Dual() : v(0.0), d(0.0) {}
  __device__ __forceinline__ Dual(double a) : v(a), d(0.0) {}
  __device__ __forceinline__ Dual(double a, double b) : v(a), d(b) {}
};

__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.v * b.d + a.d * b.v); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  double iv = 1.0 / b.v;
  double q = a.v * iv;
  return Dual(q, (a.d - q * b.d) * iv);
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return Dual(a.v + b, a.d); }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return Dual(a + b.v, b.d); }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return Dual(a.v - b, a.d); }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.d); }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
__device__ __forceinline__ Dual operator/(double a, Dual b) {
  double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
  double s = sqrt(a.v);
  return Dual(s, 0.5 * a.d / s);
}
__device__ __forceinline__ Dual dsin(Dual a) { return Dual(sin(a.v), cos(a.v) * a.d); }
__device__ __forceinline__ Dual dcos(Dual a) { return Dual(cos(a.v), -sin(a.v) * a.d); }

struct HDual {
  double v, a, b, ab;
  __device__ __forceinline__ HDual() : v(0.0), a(0.0), b(0.0), ab(0.0) {}
  __device__ __forceinline__ HDual(double x) : v(x), a(0.0), b(0.0), ab(0.0) {}
  __device__ __forceinline__ HDual(double x, double y, double z, double w) : v(x), a(y), b(z), ab(w) {}
};

// g(v + a e1 + b e2 + c e1e2) = g(v) + g'(v)(a e1 + b e2 + c e1e2) + g''(v) a b e1e2
__device__ __forceinline__ HDual hd_apply(HDual x, double g0, double g1, double g2) {
  return HDual(g0, g1 * x.a, g1 * x.b, g1 * x.ab + g2 * x.a * x.b);
}
__device__ __forceinline__ HDual operator+(HDual x, HDual y) { return HDual(x.v + y.v, x.a + y.a, x.b + y.b, x.ab + y.ab); }
__device__ __forceinline__ HDual operator-(HDual x, HDual y) { return HDual(x.v - y.v, x.a - y.a, x.b - y.b, x.ab - y.ab); }
__device__ __forceinline__ HDual operator-(HDual x) { return HDual(-x.v, -x.a, -x.b, -x.ab); }
__device__ __forceinline__ HDual operator*(HDual x, HDual y) {
  return HDual(x.v * y.v, x.v * y.a + x.a * y.v, x.v * y.b + x.b * y.v,
               x.v * y.ab + x.a * y.b + x.b * y.a + x.ab * y.v);
}
__device__ __forceinline__ HDual hd_inv(HDual y) {
  double i = 1.0 / y.v;
  return hd_apply(y, i, -i * i, 2.0 * i * i * i);
}
__device__ __forceinline__ HDual operator/(HDual x, HDual y) { return x * hd_inv(y); }
__device__ __forceinline__ HDual operator+(HDual x, double c) { return HDual(x.v + c, x.a, x.b, x.ab); }
__device__ __forceinline__ HDual operator+(double c, HDual x) { return HDual(x.v + c, x.a, x.b, x.ab); }
__device__ __forceinline__ HDual operator-(HDual x, double c) { return HDual(x.v - c, x.a, x.b, x.ab); }
__device__ __forceinline__ HDual operator-(double c, HDual x) { return HDual(c - x.v, -x.a, -x.b, -x.ab); }
__device__ __forceinline__ HDual operator*(HDual x, double c) { return HDual(x.v * c, x.a * c, x.b * c, x.ab * c); }
__device__ __forceinline__ HDual operator*(double c, HDual x) { return HDual(x.v * c, x.a * c, x.b * c, x.ab * c); }
__device__ __forceinline__ HDual operator/(HDual x, double c) { return HDual(x.v / c, x.a / c, x.b / c, x.ab / c); }
__device__ __forceinline__ HDual operator/(double c, HDual y) { return c * hd_inv(y); }
__device__ __forceinline__ HDual dsqrt(HDual x) {
  double s = sqrt(x.v);
  return hd_apply(x, s, 0.5 / s, -0.25 / (s * x.v));
}
__device__ __forceinline__ HDual dsin(HDual x) {
  double s = sin(x.v), c = cos(x.v);
  return hd_apply(x, s, c, -s);
}
__device__ __forceinline__ HDual dcos(HDual x) {
  double s = sin(x.v), c = cos(x.v);
  return hd_apply(x, c, -s, -c);
}

__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ double dsin(double a) { return sin(a); }
__device__ __forceinline__ double dcos(double a) { return cos(a); }

__device__ __forceinline__ double value_of(double a) { return a; }
__device__ __forceinline__ double value_of(Dual a) { return a.v; }
__device__ __forceinline__ double value_of(HDual a) { return a.v; }
