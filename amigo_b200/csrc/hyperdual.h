// Hyper-dual numbers for exact first and second derivatives of component
// functions on the device (Fike & Alonso, "The development of hyper-dual
// numbers for exact second-derivative calculations", AIAA 2011-886).
//
// A value a + b e1 + c e2 + d e1 e2 with e1^2 = e2^2 = 0: seeding input i
// with e1 and input j with e2, f(x) returns f in a, df/dx_i in b, df/dx_j
// in c and d2f/dx_i dx_j in d, exactly (no truncation error).  This is how
// the component derivatives that amigo generates through its A2D stacks
// (amigo/component.py:1022-1108) are obtained here for hand-written
// component functions.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define AB_HD __host__ __device__ __forceinline__
#else
#define AB_HD inline
#endif

namespace ab {

struct HD {
  double a, b, c, d;
  AB_HD HD() : a(0), b(0), c(0), d(0) {}
  AB_HD HD(double v) : a(v), b(0), c(0), d(0) {}
  AB_HD HD(double a_, double b_, double c_, double d_) : a(a_), b(b_), c(c_), d(d_) {}
};

AB_HD HD operator+(const HD& x, const HD& y) { return HD(x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d); }
AB_HD HD operator-(const HD& x, const HD& y) { return HD(x.a - y.a, x.b - y.b, x.c - y.c, x.d - y.d); }
AB_HD HD operator-(const HD& x) { return HD(-x.a, -x.b, -x.c, -x.d); }
AB_HD HD operator*(const HD& x, const HD& y) {
  return HD(x.a * y.a, x.a * y.b + x.b * y.a, x.a * y.c + x.c * y.a,
            x.a * y.d + x.b * y.c + x.c * y.b + x.d * y.a);
}
AB_HD HD operator*(double s, const HD& x) { return HD(s * x.a, s * x.b, s * x.c, s * x.d); }
AB_HD HD operator*(const HD& x, double s) { return s * x; }
AB_HD HD operator+(double s, const HD& x) { return HD(s + x.a, x.b, x.c, x.d); }
AB_HD HD operator+(const HD& x, double s) { return HD(s + x.a, x.b, x.c, x.d); }
AB_HD HD operator-(double s, const HD& x) { return HD(s - x.a, -x.b, -x.c, -x.d); }
AB_HD HD operator-(const HD& x, double s) { return HD(x.a - s, x.b, x.c, x.d); }
// 1/y: first derivative -1/y^2, second 2/y^3
AB_HD HD inv(const HD& y) {
  const double r = 1.0 / y.a, r2 = r * r;
  return HD(r, -r2 * y.b, -r2 * y.c, -r2 * y.d + 2.0 * r2 * r * y.b * y.c);
}
AB_HD HD operator/(const HD& x, const HD& y) { return x * inv(y); }
AB_HD HD operator/(const HD& x, double s) { return x * (1.0 / s); }
// Plain-double overloads so that templates over double and HD resolve
// sin/cos inside this namespace.
AB_HD double sin(double x) { return ::sin(x); }
AB_HD double cos(double x) { return ::cos(x); }
AB_HD HD sin(const HD& x) {
  const double s = ::sin(x.a), c = ::cos(x.a);
  return HD(s, c * x.b, c * x.c, c * x.d - s * x.b * x.c);
}
AB_HD HD cos(const HD& x) {
  const double s = ::sin(x.a), c = ::cos(x.a);
  return HD(c, -s * x.b, -s * x.c, -s * x.d - c * x.b * x.c);
}

}  // namespace ab
