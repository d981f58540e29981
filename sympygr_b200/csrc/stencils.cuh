// Finite-difference line operators of the reference's default build, evaluated on
// values staged in shared memory.
//
//   line_d1 : deriv64_{x,y,z}    bssn/src/derivs.cpp:2055-2434  6th-order centred first
//                                                               derivative, 4th-order closures
//   line_d2 : deriv64_{xx,yy,zz} bssn/src/derivs.cpp:2443-2833  6th-order centred second
//                                                               derivative, 4th-order closures
//   line_ko : ko_deriv42_{x,y,z} bssn/src/derivs.cpp:915-1319   Kreiss-Oliger operator
//
// Each takes a pointer `p` to the value at the evaluation point, the element stride
// `s` along the operator axis, the point's padded index `pos` on that axis, the
// padded extent `n`, and whether the low/high face of that axis is a domain
// boundary (bflag bits).  Closure rows replace the centred row within three points
// of a flagged face; the high side wins where both apply, as the reference runs
// its LEFT loop before its RIGHT loop.  Closure rows reach up to four points
// inward; callers stage a 4-point halo.
//
// Rounding: every product and sum is an explicitly rounded IEEE operation
// (__dmul_rn/__dadd_rn, never contracted into an FMA) taken in the reference's
// left-to-right order, so each stencil value equals the reference's bit for bit.
// The stencils cancel terms of size 10^2 |u| down to h|u'|; with contraction the
// last bits of a first derivative move, and composing two closure rows on a block
// edge (D_y of D_x) amplifies that to ~1e-12 of the field's range.
#pragma once

namespace b200bssn {

struct LineScales {
  double d1_c, d1_b;   // idx/60, idx/12                      (derivs.cpp:2059-2061)
  double d2_c, d2_b;   // idx^2/180, idx^2/12                 (derivs.cpp:2447-2449)
  double ko_c;         // -1/64/dx                            (derivs.cpp:919)
  double ko_s1, ko_s2, ko_s3;  // 49/48*64*dx, 43/48*64*dx, 59/48*64*dx (:921-923)
  double adv_b2;       // 0.5*idx (upwind rows /2h; the /12h rows use d1_b, derivs.cpp:499-501)
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
  c.adv_b2 = 0.50 * ih;
  return c;
}

// 4th-order upwind advective derivative (bssn/src/derivs.cpp:495-900, the upwind operator
// of the reference's 4th-order build).  Row ids, with offsets from the point in the
// reference's summation order:
//   0  centre, beta > 0 : (-3 u-1 - 10 u0 + 18 u1 - 6 u2 + u3) / 12h
//   1  centre, otherwise: (-u-3 + 6 u-2 - 18 u-1 + 10 u0 + 3 u1) / 12h
//   2  (-3 u0 + 4 u1 - u2) / 2h     3  (-u-1 + u1) / 2h     4  (u-2 - 4 u-1 + 3 u0) / 2h
// On a flagged low face the points 3, 4, 5 use rows 2, 2|3, 0|4 (beta > 0 | otherwise;
// derivs.cpp:538-575) and on a flagged high face the points n-6, n-5, n-4 use rows 2|1,
// 3|4, 4 (derivs.cpp:577-620).  Every row reaches at most three points from the point.
__host__ __device__ inline int adv_row_id(int pos, int n, bool lo, bool hi, bool up) {
  if (hi && pos >= n - 6) {
    const int r = pos - (n - 6);
    return r == 0 ? (up ? 2 : 1) : (r == 1 ? (up ? 3 : 4) : 4);
  }
  if (lo && pos < 6) {
    const int r = pos - 3;
    return r == 0 ? 2 : (r == 1 ? (up ? 2 : 3) : (up ? 0 : 4));
  }
  return up ? 0 : 1;
}

// acc + c*v with both operations rounded separately
__device__ __forceinline__ double mad_rn(double acc, double c, double v) {
  return __dadd_rn(acc, __dmul_rn(c, v));
}

// Sum of coefficient[k] * value(offset[k]) in the given order (first term c0*v0).
#define B2_T(c, k) __dmul_rn((c), p[(k) * s])
#define B2_Q(c, k) __dmul_rn((c), q[(k) * s])

__device__ __forceinline__ double line_d1(const double* p, int s, int pos, int n, bool lo,
                                          bool hi, const LineScales& c) {
  if (hi && pos >= n - 6) {
    const int r = pos - (n - 6);
    const double* q = p + (n - 4 - pos) * s;  // value at ie-1 = n-4; derivs.cpp:2132-2155
    double a;
    if (r == 0) {
      a = B2_Q(1.0, -4);
      a = __dadd_rn(a, B2_Q(-8.0, -3));
      a = __dadd_rn(a, B2_Q(8.0, -1));
      a = __dadd_rn(a, B2_Q(-1.0, 0));
    } else if (r == 1) {
      a = B2_Q(-1.0, -4);
      a = __dadd_rn(a, B2_Q(6.0, -3));
      a = __dadd_rn(a, B2_Q(-18.0, -2));
      a = __dadd_rn(a, B2_Q(10.0, -1));
      a = __dadd_rn(a, B2_Q(3.0, 0));
    } else {
      a = B2_Q(3.0, -4);
      a = __dadd_rn(a, B2_Q(-16.0, -3));
      a = __dadd_rn(a, B2_Q(36.0, -2));
      a = __dadd_rn(a, B2_Q(-48.0, -1));
      a = __dadd_rn(a, B2_Q(25.0, 0));
    }
    return __dmul_rn(a, c.d1_b);
  }
  if (lo && pos < 6) {
    const int r = pos - 3;
    const double* q = p - r * s;  // value at index 3; derivs.cpp:2094-2115
    double a;
    if (r == 0) {
      a = B2_Q(-25.0, 0);
      a = __dadd_rn(a, B2_Q(48.0, 1));
      a = __dadd_rn(a, B2_Q(-36.0, 2));
      a = __dadd_rn(a, B2_Q(16.0, 3));
      a = __dadd_rn(a, B2_Q(-3.0, 4));
    } else if (r == 1) {
      a = B2_Q(-3.0, 0);
      a = __dadd_rn(a, B2_Q(-10.0, 1));
      a = __dadd_rn(a, B2_Q(18.0, 2));
      a = __dadd_rn(a, B2_Q(-6.0, 3));
      a = __dadd_rn(a, B2_Q(1.0, 4));
    } else {
      a = B2_Q(1.0, 0);
      a = __dadd_rn(a, B2_Q(-8.0, 1));
      a = __dadd_rn(a, B2_Q(8.0, 3));
      a = __dadd_rn(a, B2_Q(-1.0, 4));
    }
    return __dmul_rn(a, c.d1_b);
  }
  double a = B2_T(-1.0, -3);
  a = __dadd_rn(a, B2_T(9.0, -2));
  a = __dadd_rn(a, B2_T(-45.0, -1));
  a = __dadd_rn(a, B2_T(45.0, 1));
  a = __dadd_rn(a, B2_T(-9.0, 2));
  a = __dadd_rn(a, B2_T(1.0, 3));
  return __dmul_rn(a, c.d1_c);
}

__device__ __forceinline__ double line_d2(const double* p, int s, int pos, int n, bool lo,
                                          bool hi, const LineScales& c) {
  if (hi && pos >= n - 6) {
    const int r = pos - (n - 6);
    const double* q = p + (n - 4 - pos) * s;  // derivs.cpp:2530-2551
    double a;
    if (r == 0) {
      a = B2_Q(-1.0, -4);
      a = __dadd_rn(a, B2_Q(16.0, -3));
      a = __dadd_rn(a, B2_Q(-30.0, -2));
      a = __dadd_rn(a, B2_Q(16.0, -1));
      a = __dadd_rn(a, B2_Q(-1.0, 0));
    } else if (r == 1) {
      a = B2_Q(-1.0, -4);
      a = __dadd_rn(a, B2_Q(4.0, -3));
      a = __dadd_rn(a, B2_Q(6.0, -2));
      a = __dadd_rn(a, B2_Q(-20.0, -1));
      a = __dadd_rn(a, B2_Q(11.0, 0));
    } else {
      a = B2_Q(11.0, -4);
      a = __dadd_rn(a, B2_Q(-56.0, -3));
      a = __dadd_rn(a, B2_Q(114.0, -2));
      a = __dadd_rn(a, B2_Q(-104.0, -1));
      a = __dadd_rn(a, B2_Q(35.0, 0));
    }
    return __dmul_rn(a, c.d2_b);
  }
  if (lo && pos < 6) {
    const int r = pos - 3;
    const double* q = p - r * s;  // derivs.cpp:2490-2510
    double a;
    if (r == 0) {
      a = B2_Q(35.0, 0);
      a = __dadd_rn(a, B2_Q(-104.0, 1));
      a = __dadd_rn(a, B2_Q(114.0, 2));
      a = __dadd_rn(a, B2_Q(-56.0, 3));
      a = __dadd_rn(a, B2_Q(11.0, 4));
    } else if (r == 1) {
      a = B2_Q(11.0, 0);
      a = __dadd_rn(a, B2_Q(-20.0, 1));
      a = __dadd_rn(a, B2_Q(6.0, 2));
      a = __dadd_rn(a, B2_Q(4.0, 3));
      a = __dadd_rn(a, B2_Q(-1.0, 4));
    } else {
      a = B2_Q(-1.0, 0);
      a = __dadd_rn(a, B2_Q(16.0, 1));
      a = __dadd_rn(a, B2_Q(-30.0, 2));
      a = __dadd_rn(a, B2_Q(16.0, 3));
      a = __dadd_rn(a, B2_Q(-1.0, 4));
    }
    return __dmul_rn(a, c.d2_b);
  }
  double a = B2_T(2.0, -3);
  a = __dadd_rn(a, B2_T(-27.0, -2));
  a = __dadd_rn(a, B2_T(270.0, -1));
  a = __dadd_rn(a, B2_T(-490.0, 0));
  a = __dadd_rn(a, B2_T(270.0, 1));
  a = __dadd_rn(a, B2_T(-27.0, 2));
  a = __dadd_rn(a, B2_T(2.0, 3));
  return __dmul_rn(a, c.d2_c);
}

__device__ __forceinline__ double line_ko(const double* p, int s, int pos, int n, bool lo,
                                          bool hi, const LineScales& c) {
  if (hi && pos >= n - 6) {
    const int r = pos - (n - 6);
    const double* q = p + (n - 4 - pos) * s;  // derivs.cpp:1006-1028
    double a;
    if (r == 0) {
      a = q[-5 * s];
      a = __dadd_rn(a, B2_Q(-6.0, -4));
      a = __dadd_rn(a, B2_Q(15.0, -3));
      a = __dadd_rn(a, B2_Q(-19.0, -2));
      a = __dadd_rn(a, B2_Q(12.0, -1));
      a = __dadd_rn(a, B2_Q(-3.0, 0));
      return __ddiv_rn(a, c.ko_s1);
    } else if (r == 1) {
      a = q[-4 * s];
      a = __dadd_rn(a, B2_Q(-6.0, -3));
      a = __dadd_rn(a, B2_Q(12.0, -2));
      a = __dadd_rn(a, B2_Q(-10.0, -1));
      a = __dadd_rn(a, B2_Q(3.0, 0));
      return __ddiv_rn(a, c.ko_s2);
    }
    a = q[-3 * s];
    a = __dadd_rn(a, B2_Q(-3.0, -2));
    a = __dadd_rn(a, B2_Q(3.0, -1));
    a = __dsub_rn(a, q[0]);
    return __ddiv_rn(a, c.ko_s3);
  }
  if (lo && pos < 6) {
    const int r = pos - 3;
    const double* q = p - r * s;  // derivs.cpp:969-990 (summed from the far point inwards)
    double a;
    if (r == 0) {
      a = q[3 * s];
      a = __dadd_rn(a, B2_Q(-3.0, 2));
      a = __dadd_rn(a, B2_Q(3.0, 1));
      a = __dsub_rn(a, q[0]);
      return __ddiv_rn(a, c.ko_s3);
    } else if (r == 1) {
      a = q[4 * s];
      a = __dadd_rn(a, B2_Q(-6.0, 3));
      a = __dadd_rn(a, B2_Q(12.0, 2));
      a = __dadd_rn(a, B2_Q(-10.0, 1));
      a = __dadd_rn(a, B2_Q(3.0, 0));
      return __ddiv_rn(a, c.ko_s2);
    }
    a = q[5 * s];
    a = __dadd_rn(a, B2_Q(-6.0, 4));
    a = __dadd_rn(a, B2_Q(15.0, 3));
    a = __dadd_rn(a, B2_Q(-19.0, 2));
    a = __dadd_rn(a, B2_Q(12.0, 1));
    a = __dadd_rn(a, B2_Q(-3.0, 0));
    return __ddiv_rn(a, c.ko_s1);
  }
  double a = -p[-3 * s];
  a = __dadd_rn(a, B2_T(6.0, -2));
  a = __dadd_rn(a, B2_T(-15.0, -1));
  a = __dadd_rn(a, B2_T(20.0, 0));
  a = __dadd_rn(a, B2_T(-15.0, 1));
  a = __dadd_rn(a, B2_T(6.0, 2));
  a = __dsub_rn(a, p[3 * s]);
  return __dmul_rn(c.ko_c, a);
}

#undef B2_T
#undef B2_Q

// Centred rows on a register window w[] (C = index of the evaluation point).
// Callers invoke these inside fully unrolled loops, so every index folds to a
// constant and the window stays in registers.  Same operations and order as the
// centred branches above.
template <int N>
__device__ __forceinline__ double win_d1(const double (&w)[N], const int C,
                                         const LineScales& c) {
  double a = __dmul_rn(-1.0, w[C - 3]);
  a = mad_rn(a, 9.0, w[C - 2]);
  a = mad_rn(a, -45.0, w[C - 1]);
  a = mad_rn(a, 45.0, w[C + 1]);
  a = mad_rn(a, -9.0, w[C + 2]);
  a = mad_rn(a, 1.0, w[C + 3]);
  return __dmul_rn(a, c.d1_c);
}

template <int N>
__device__ __forceinline__ double win_d2(const double (&w)[N], const int C,
                                         const LineScales& c) {
  double a = __dmul_rn(2.0, w[C - 3]);
  a = mad_rn(a, -27.0, w[C - 2]);
  a = mad_rn(a, 270.0, w[C - 1]);
  a = mad_rn(a, -490.0, w[C]);
  a = mad_rn(a, 270.0, w[C + 1]);
  a = mad_rn(a, -27.0, w[C + 2]);
  a = mad_rn(a, 2.0, w[C + 3]);
  return __dmul_rn(a, c.d2_c);
}

template <int N>
__device__ __forceinline__ double win_ko(const double (&w)[N], const int C,
                                         const LineScales& c) {
  double a = -w[C - 3];
  a = mad_rn(a, 6.0, w[C - 2]);
  a = mad_rn(a, -15.0, w[C - 1]);
  a = mad_rn(a, 20.0, w[C]);
  a = mad_rn(a, -15.0, w[C + 1]);
  a = mad_rn(a, 6.0, w[C + 2]);
  a = __dsub_rn(a, w[C + 3]);
  return __dmul_rn(c.ko_c, a);
}

// True when the point at padded index `pos` takes a closure row.
__device__ __forceinline__ bool closure_row(int pos, int n, bool lo, bool hi) {
  return (lo && pos < 6) || (hi && pos >= n - 6);
}

}  // namespace b200bssn
