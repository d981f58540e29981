// Finite-difference line operators of the reference's default build, evaluated on
// values staged in shared memory.
//
//   d1  : deriv64_{x,y,z}   bssn/src/derivs.cpp:2055-2434  6th-order centred first
//                                                          derivative, 4th-order closures
//   d2  : deriv64_{xx,yy,zz} bssn/src/derivs.cpp:2443-2833 6th-order centred second
//                                                          derivative, 4th-order closures
//   ko  : ko_deriv42_{x,y,z} bssn/src/derivs.cpp:915-1319  Kreiss-Oliger operator
//
// Each takes a pointer `p` to the value at the evaluation point, the element stride
// `s` along the operator axis, the point's padded index `pos` on that axis, the
// padded extent `n`, and whether the low/high face of that axis is a domain
// boundary (bflag bits).  Closure rows replace the centred row within three points
// of a flagged face; the high side wins where both apply, as the reference runs
// its LEFT loop before its RIGHT loop.  Terms are summed in the reference's order.
// Closure rows reach up to four points inward; callers stage a 4-point halo.
#pragma once

namespace b200bssn {

struct LineScales {
  double d1_c, d1_b;   // idx/60, idx/12                      (derivs.cpp:2059-2061)
  double d2_c, d2_b;   // idx^2/180, idx^2/12                 (derivs.cpp:2447-2449)
  double ko_c;         // -1/64/dx                            (derivs.cpp:919)
  double ko_s1, ko_s2, ko_s3;  // 49/48*64*dx, 43/48*64*dx, 59/48*64*dx (:921-923)
};

__host__ __device__ inline LineScales make_line_scales(double h) {
  LineScales c;
  const double ih = 1.0 / h;
  c.d1_c = ih / 60.0;
  c.d1_b = ih / 12.0;
  const double ih2 = 1.0 / (h * h);
  c.d2_c = ih2 / 180.0;
  c.d2_b = ih2 / 12.0;
  c.ko_c = -1.0 / 64.0 / h;
  c.ko_s3 = 59.0 / 48.0 * 64 * h;
  c.ko_s2 = 43.0 / 48.0 * 64 * h;
  c.ko_s1 = 49.0 / 48.0 * 64 * h;
  return c;
}

#define B2_AT(k) p[(k) * s]

__device__ __forceinline__ double line_d1(const double* p, int s, int pos, int n, bool lo,
                                          bool hi, const LineScales& c) {
  if (hi && pos >= n - 6) {
    const int r = pos - (n - 6);
    // q = value at index n-4 (ie-1); rows of derivs.cpp:2132-2155
    const double* q = p + (n - 4 - pos) * s;
#define Q(k) q[(k) * s]
    if (r == 0) return (1.0 * Q(-4) - 8.0 * Q(-3) + 8.0 * Q(-1) - 1.0 * Q(0)) * c.d1_b;
    if (r == 1) return (-1.0 * Q(-4) + 6.0 * Q(-3) - 18.0 * Q(-2) + 10.0 * Q(-1) + 3.0 * Q(0)) * c.d1_b;
    return (3.0 * Q(-4) - 16.0 * Q(-3) + 36.0 * Q(-2) - 48.0 * Q(-1) + 25.0 * Q(0)) * c.d1_b;
#undef Q
  }
  if (lo && pos < 6) {
    const int r = pos - 3;
    const double* q = p - r * s;  // value at index 3; rows of derivs.cpp:2094-2115
#define Q(k) q[(k) * s]
    if (r == 0) return (-25.0 * Q(0) + 48.0 * Q(1) - 36.0 * Q(2) + 16.0 * Q(3) - 3.0 * Q(4)) * c.d1_b;
    if (r == 1) return (-3.0 * Q(0) - 10.0 * Q(1) + 18.0 * Q(2) - 6.0 * Q(3) + 1.0 * Q(4)) * c.d1_b;
    return (1.0 * Q(0) - 8.0 * Q(1) + 8.0 * Q(3) - 1.0 * Q(4)) * c.d1_b;
#undef Q
  }
  return (-1.0 * B2_AT(-3) + 9.0 * B2_AT(-2) - 45.0 * B2_AT(-1) + 45.0 * B2_AT(1) -
          9.0 * B2_AT(2) + 1.0 * B2_AT(3)) * c.d1_c;
}

__device__ __forceinline__ double line_d2(const double* p, int s, int pos, int n, bool lo,
                                          bool hi, const LineScales& c) {
  if (hi && pos >= n - 6) {
    const int r = pos - (n - 6);
    const double* q = p + (n - 4 - pos) * s;  // derivs.cpp:2530-2551
#define Q(k) q[(k) * s]
    if (r == 0) return (-1.0 * Q(-4) + 16.0 * Q(-3) - 30.0 * Q(-2) + 16.0 * Q(-1) - 1.0 * Q(0)) * c.d2_b;
    if (r == 1) return (-1.0 * Q(-4) + 4.0 * Q(-3) + 6.0 * Q(-2) - 20.0 * Q(-1) + 11.0 * Q(0)) * c.d2_b;
    return (11.0 * Q(-4) - 56.0 * Q(-3) + 114.0 * Q(-2) - 104.0 * Q(-1) + 35.0 * Q(0)) * c.d2_b;
#undef Q
  }
  if (lo && pos < 6) {
    const int r = pos - 3;
    const double* q = p - r * s;  // derivs.cpp:2490-2510
#define Q(k) q[(k) * s]
    if (r == 0) return (35.0 * Q(0) - 104.0 * Q(1) + 114.0 * Q(2) - 56.0 * Q(3) + 11.0 * Q(4)) * c.d2_b;
    if (r == 1) return (11.0 * Q(0) - 20.0 * Q(1) + 6.0 * Q(2) + 4.0 * Q(3) - 1.0 * Q(4)) * c.d2_b;
    return (-1.0 * Q(0) + 16.0 * Q(1) - 30.0 * Q(2) + 16.0 * Q(3) - 1.0 * Q(4)) * c.d2_b;
#undef Q
  }
  return (2.0 * B2_AT(-3) - 27.0 * B2_AT(-2) + 270.0 * B2_AT(-1) - 490.0 * B2_AT(0) +
          270.0 * B2_AT(1) - 27.0 * B2_AT(2) + 2.0 * B2_AT(3)) * c.d2_c;
}

__device__ __forceinline__ double line_ko(const double* p, int s, int pos, int n, bool lo,
                                          bool hi, const LineScales& c) {
  if (hi && pos >= n - 6) {
    const int r = pos - (n - 6);
    const double* q = p + (n - 4 - pos) * s;  // derivs.cpp:1006-1028
#define Q(k) q[(k) * s]
    if (r == 0) return (Q(-5) - 6.0 * Q(-4) + 15.0 * Q(-3) - 19.0 * Q(-2) + 12.0 * Q(-1) - 3.0 * Q(0)) / c.ko_s1;
    if (r == 1) return (Q(-4) - 6.0 * Q(-3) + 12.0 * Q(-2) - 10.0 * Q(-1) + 3.0 * Q(0)) / c.ko_s2;
    return (Q(-3) - 3.0 * Q(-2) + 3.0 * Q(-1) - Q(0)) / c.ko_s3;
#undef Q
  }
  if (lo && pos < 6) {
    const int r = pos - 3;
    const double* q = p - r * s;  // derivs.cpp:969-990
#define Q(k) q[(k) * s]
    if (r == 0) return (Q(3) - 3.0 * Q(2) + 3.0 * Q(1) - Q(0)) / c.ko_s3;
    if (r == 1) return (Q(4) - 6.0 * Q(3) + 12.0 * Q(2) - 10.0 * Q(1) + 3.0 * Q(0)) / c.ko_s2;
    return (Q(5) - 6.0 * Q(4) + 15.0 * Q(3) - 19.0 * Q(2) + 12.0 * Q(1) - 3.0 * Q(0)) / c.ko_s1;
#undef Q
  }
  return c.ko_c * (-B2_AT(-3) + 6.0 * B2_AT(-2) - 15.0 * B2_AT(-1) + 20.0 * B2_AT(0) -
                   15.0 * B2_AT(1) + 6.0 * B2_AT(2) - B2_AT(3));
}

#undef B2_AT

}  // namespace b200bssn
