// The kernels of one right-hand-side evaluation of a chunk of blocks.
//
//  derivative stage     a CTA streams one variable along z through one 16x8 column
//                       tile of a unit and writes, per interior point, the
//                       variable's first derivatives, its second derivatives when
//                       it has them (mixed ones as compositions D_y(D_x u),
//                       D_z(D_x u), D_z(D_y u), exactly as
//                       bssn/scripts/bssnrhs_derivs.h composes them), and the sum
//                       of its three KO terms, into the chunk's derivative scratch:
//                       bssn_derivs_kind_kernel (two persistent kernels, variables
//                       without / with second derivatives; the plan path) or
//                       bssn_derivs_kernel (all 24 variables; the allocation-free
//                       entry point).
//  algebra stage        per interior point the generated BSSN algebra (or, on a
//                       flagged face plane, the Sommerfeld value of
//                       bssn/src/rhs.cpp:833-977), plus sigma times the KO sum
//                       (bssn/src/rhs.cpp:332-369), written to the RHS arrays -- or,
//                       in an RK4 stage, folded straight into the stage update (see
//                       RkStage) so the RHS never goes to memory:
//                       bssn_algebra_staged_kernel (persistent warps reading their
//                       points' scratch from shared memory; the plan path) or
//                       bssn_algebra_kernel (one CTA per 128-point run; the
//                       allocation-free entry point).
#pragma once
#include <stdint.h>

#include "generated/bssn_rhs_algebra.cuh"
#include "generated/bssn_rhs_algebra_adv.cuh"
#include "generated/bssn_rhs_algebra_split.cuh"
#include "plan_types.h"
#include "stencils.cuh"

namespace b200bssn {


// VAR index -> position in the second-derivative list (gt0..gt5, chi, alpha,
// beta0..2; bssn/scripts/gen_bssnrhs_code:31-32), -1 if none.
__device__ __forceinline__ int dd_index(int v) {
  switch (v) {
    case 12: return 0; case 13: return 1; case 14: return 2;
    case 15: return 3; case 16: return 4; case 17: return 5;
    case 1: return 6;  case 0: return 7;
    case 6: return 8;  case 7: return 9;  case 8: return 10;
    default: return -1;
  }
}

struct DerivArgs {
  const double* u[kNumVars];
  const BlockDev* blocks;
  const UnitDev* units;
  const TileDev* tiles;
  void* dscr;        // NS derivative slots (double or float), layout scr_index
  void* koscr;       // kNumVars KO sums (double or float, like dscr), layout scr_index
  int32_t cap;       // points per slot (multiple of 32); NS * cap < 2^31: 32-bit offsets
  int32_t tile_base;
  int32_t tile_count;
  int* counter;      // work counter of this launch, zero at launch
};

// ---------------------------------------------------------------------------
// Derivative kernel: a 2.5-D streaming stencil.
//
// A work item is one 16x8 column tile of a unit (a z-slab of up to 48 interior
// planes of one block) and one variable; the CTA marches along z.  Each z step
// brings one plane of the tile plus its 4-point x-y halo into shared memory
// (cp.async into four plane buffers: three planes stream in while one is
// differentiated).  In-plane derivatives (D_x, D_y, D_xx, D_yy, D_y(D_x), ko_x,
// ko_y) come from that plane; the z derivatives of the variable and of its D_x
// and D_y (D_z, D_zz, ko_z, D_z(D_x), D_z(D_y)) come from register queues that
// each thread keeps for its own column (9 planes deep where a closure row may reach
// 4 planes, else 7), so every plane is loaded once per variable and no z halo is
// recomputed.  The item's code is instantiated for variables with and without
// second derivatives (DD), so the 13 variables that need only first derivatives and
// KO carry no D_x/D_y queues or halo rows, and for items with and without closure
// rows (CL), so the items away from flagged faces carry no closure tests.
// ---------------------------------------------------------------------------
constexpr int kPlaneW = kTileX + 2 * kHalo;  // 24: plane width incl. halo
constexpr int kPlaneH = kTileY + 2 * kHalo;  // 16
constexpr int kPlane = kPlaneW * kPlaneH;     // doubles per staged plane
constexpr int kDxRows = kTileY + 2 * kHalo;  // D_x rows kept per plane (y halo)
constexpr int kQ = 2 * kHalo + 1;            // z queue depth (planes z-4 .. z+4)
static_assert(kTileX == 16 && kDerivThreads == kTileX * kTileY && kTileY <= 16, "one thread per tile column");
// plane copy: each warp stages every (kDerivThreads / 32)-th row of the plane
constexpr int kStageRows = kPlaneH / (kDerivThreads / 32);
static_assert(kStageRows * (kDerivThreads / 32) == kPlaneH, "plane rows split evenly over the warps");
static_assert(kDxRows <= 2 * kTileY, "two D_x halo rows per thread cover the plane");

// Shape of a derivative CTA for tiles of 16 x TY columns (TY = 4, 8 or 16): one thread
// per column, the staged plane with its 4-point halo, the y-halo D_x rows.
template <int TY>
struct TileShape {
  static constexpr int kThreads = kTileX * TY;
  static constexpr int kWarps = kThreads / 32;
  static constexpr int kPlaneH = TY + 2 * kHalo;
  static constexpr int kPlane = kPlaneW * kPlaneH;
  static constexpr int kDxRows = TY + 2 * kHalo;
  static constexpr int kDxPerThread = (kDxRows + TY - 1) / TY;  // D_x halo rows per thread
  static constexpr int kStageRows = kPlaneH / kWarps;           // plane rows per thread
  static_assert(kStageRows * kWarps == kPlaneH, "plane rows split evenly over the warps");
};

// the copy is issued only when `p` holds; otherwise nothing is read or written
__device__ __forceinline__ void cp_async8_if(double* smem_dst, const double* gmem_src, bool p) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile(
      "{\n .reg .pred q;\n setp.ne.b32 q, %2, 0;\n @q cp.async.ca.shared.global [%0], [%1], 8;\n}\n" ::"r"(s),
      "l"(gmem_src), "r"((int)p)
      : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Z-direction rows on a queue q[0..8] holding planes zo-4 .. zo+4 of one column.
// `zc` selects the row: -1 centred, 0..2 the low-side closure rows (zo = 3,4,5),
// 3..5 the high-side rows (zo = n-6, n-5, n-4); indices are compile-time in every
// case, so the queue stays in registers.  Same operations and order as line_*;
// values are widened to double (exact for double queues).
__device__ __forceinline__ int z_case(int zo, int n, bool lo, bool hi) {
  if (hi && zo >= n - 6) return 3 + (zo - (n - 6));
  if (lo && zo < 6) return zo - 3;
  return -1;
}

#define ZQ(k) ((double)q[(k)])
template <typename T>
__device__ __forceinline__ double zq_d1_closure(const T (&q)[kQ], int zc, const LineScales& c) {
  double a;
  switch (zc) {
    case 0:  // zo=3: planes 3..7 -> q[4..8]
      a = __dmul_rn(-25.0, ZQ(4)); a = mad_rn(a, 48.0, ZQ(5)); a = mad_rn(a, -36.0, ZQ(6));
      a = mad_rn(a, 16.0, ZQ(7)); a = mad_rn(a, -3.0, ZQ(8));
      break;
    case 1:  // zo=4: planes 3..7 -> q[3..7]
      a = __dmul_rn(-3.0, ZQ(3)); a = mad_rn(a, -10.0, ZQ(4)); a = mad_rn(a, 18.0, ZQ(5));
      a = mad_rn(a, -6.0, ZQ(6)); a = mad_rn(a, 1.0, ZQ(7));
      break;
    case 2:  // zo=5: planes 3,4,6,7 -> q[2,3,5,6]
    case 3:  // zo=n-6: planes n-8,n-7,n-5,n-4 -> q[2,3,5,6]
      a = __dmul_rn(1.0, ZQ(2)); a = mad_rn(a, -8.0, ZQ(3)); a = mad_rn(a, 8.0, ZQ(5));
      a = mad_rn(a, -1.0, ZQ(6));
      break;
    case 4:  // zo=n-5: planes n-8..n-4 -> q[1..5]
      a = __dmul_rn(-1.0, ZQ(1)); a = mad_rn(a, 6.0, ZQ(2)); a = mad_rn(a, -18.0, ZQ(3));
      a = mad_rn(a, 10.0, ZQ(4)); a = mad_rn(a, 3.0, ZQ(5));
      break;
    default:  // 5: zo=n-4: planes n-8..n-4 -> q[0..4]
      a = __dmul_rn(3.0, ZQ(0)); a = mad_rn(a, -16.0, ZQ(1)); a = mad_rn(a, 36.0, ZQ(2));
      a = mad_rn(a, -48.0, ZQ(3)); a = mad_rn(a, 25.0, ZQ(4));
      break;
  }
  return __dmul_rn(a, c.d1_b);
}

template <typename T>
__device__ __forceinline__ double zq_d2_closure(const T (&q)[kQ], int zc, const LineScales& c) {
  double a;
  switch (zc) {
    case 0:
      a = __dmul_rn(35.0, ZQ(4)); a = mad_rn(a, -104.0, ZQ(5)); a = mad_rn(a, 114.0, ZQ(6));
      a = mad_rn(a, -56.0, ZQ(7)); a = mad_rn(a, 11.0, ZQ(8));
      break;
    case 1:
      a = __dmul_rn(11.0, ZQ(3)); a = mad_rn(a, -20.0, ZQ(4)); a = mad_rn(a, 6.0, ZQ(5));
      a = mad_rn(a, 4.0, ZQ(6)); a = mad_rn(a, -1.0, ZQ(7));
      break;
    case 2:
    case 3:
      a = __dmul_rn(-1.0, ZQ(2)); a = mad_rn(a, 16.0, ZQ(3)); a = mad_rn(a, -30.0, ZQ(4));
      a = mad_rn(a, 16.0, ZQ(5)); a = mad_rn(a, -1.0, ZQ(6));
      break;
    case 4:
      a = __dmul_rn(-1.0, ZQ(1)); a = mad_rn(a, 4.0, ZQ(2)); a = mad_rn(a, 6.0, ZQ(3));
      a = mad_rn(a, -20.0, ZQ(4)); a = mad_rn(a, 11.0, ZQ(5));
      break;
    default:
      a = __dmul_rn(11.0, ZQ(0)); a = mad_rn(a, -56.0, ZQ(1)); a = mad_rn(a, 114.0, ZQ(2));
      a = mad_rn(a, -104.0, ZQ(3)); a = mad_rn(a, 35.0, ZQ(4));
      break;
  }
  return __dmul_rn(a, c.d2_b);
}

template <typename T>
__device__ __forceinline__ double zq_ko_closure(const T (&q)[kQ], int zc, const LineScales& c) {
  double a;
  switch (zc) {
    case 0:  // (u6 - 3u5 + 3u4 - u3)/s3, planes 3..6 -> q[4..7]
      a = ZQ(7); a = mad_rn(a, -3.0, ZQ(6)); a = mad_rn(a, 3.0, ZQ(5)); a = __dsub_rn(a, ZQ(4));
      return __ddiv_rn(a, c.ko_s3);
    case 1:  // planes 3..7 -> q[3..7]
      a = ZQ(7); a = mad_rn(a, -6.0, ZQ(6)); a = mad_rn(a, 12.0, ZQ(5)); a = mad_rn(a, -10.0, ZQ(4));
      a = mad_rn(a, 3.0, ZQ(3));
      return __ddiv_rn(a, c.ko_s2);
    case 2:  // planes 3..8 -> q[2..7]
      a = ZQ(7); a = mad_rn(a, -6.0, ZQ(6)); a = mad_rn(a, 15.0, ZQ(5)); a = mad_rn(a, -19.0, ZQ(4));
      a = mad_rn(a, 12.0, ZQ(3)); a = mad_rn(a, -3.0, ZQ(2));
      return __ddiv_rn(a, c.ko_s1);
    case 3:  // zo=n-6: planes n-9..n-4 -> q[1..6]
      a = ZQ(1); a = mad_rn(a, -6.0, ZQ(2)); a = mad_rn(a, 15.0, ZQ(3)); a = mad_rn(a, -19.0, ZQ(4));
      a = mad_rn(a, 12.0, ZQ(5)); a = mad_rn(a, -3.0, ZQ(6));
      return __ddiv_rn(a, c.ko_s1);
    case 4:  // zo=n-5: planes n-8..n-4 -> q[1..5]
      a = ZQ(1); a = mad_rn(a, -6.0, ZQ(2)); a = mad_rn(a, 12.0, ZQ(3)); a = mad_rn(a, -10.0, ZQ(4));
      a = mad_rn(a, 3.0, ZQ(5));
      return __ddiv_rn(a, c.ko_s2);
    default:  // 5: zo=n-4: planes n-7..n-4 -> q[1..4]
      a = ZQ(1); a = mad_rn(a, -3.0, ZQ(2)); a = mad_rn(a, 3.0, ZQ(3)); a = __dsub_rn(a, ZQ(4));
      return __ddiv_rn(a, c.ko_s3);
  }
}
#undef ZQ

// z rows of an item on its queue q (planes zo-N/2 .. zo+N/2): with closures (CL, N =
// kQ) the closure row `zc` where zc >= 0, else the centred row
template <bool CL, class Rows, typename T, int N>
__device__ __forceinline__ double zrow_d1(const T (&q)[N], int zc, const LineScales& c) {
  if constexpr (CL) {
    if (zc >= 0) return zq_d1_closure(q, zc, c);
  }
  return (double)Rows::d1(q, N / 2, c);
}
template <bool CL, class Rows, typename T, int N>
__device__ __forceinline__ double zrow_d2(const T (&q)[N], int zc, const LineScales& c) {
  if constexpr (CL) {
    if (zc >= 0) return zq_d2_closure(q, zc, c);
  }
  return (double)Rows::d2(q, N / 2, c);
}
template <bool CL, class Rows, typename T, int N>
__device__ __forceinline__ double zrow_ko(const T (&q)[N], int zc, const LineScales& c) {
  if constexpr (CL) {
    if (zc >= 0) return zq_ko_closure(q, zc, c);
  }
  return Rows::ko(q, N / 2, c);
}

template <typename T, int N>
__device__ __forceinline__ void q_push(T (&q)[N], T v) {
#pragma unroll
  for (int k = 0; k < N - 1; ++k) q[k] = q[k + 1];
  q[N - 1] = v;
}

// Centred-row arithmetic of the derivative kernel, by precision mode.
//
// ExactRows (FP64 mode): the reference's operations and order, each rounded
// (the win_* rows), so every derivative equals the reference's bit for bit.
//
// SplitRows (MIXED mode): the split-precision stencil.  Neighbour values enter
// only through FP64 differences taken before any downcast -- antisymmetric
// a_k = u(+k) - u(-k) for first derivatives, symmetric s_k = u(+k) + u(-k) - 2u
// for second derivatives (the centre weight cancels exactly since the weights
// sum to zero) -- whose weighted sum (fused multiply-adds allowed) is rounded once
// to FP32, the precision the derivative is stored in.  The Kreiss-Oliger row, a
// sixth difference that cancels all lower orders, stays in FP64 (from the same
// symmetric sums).
struct ExactRows {
  using D = double;
  template <typename T, int N>
  static __device__ __forceinline__ D d1(const T (&w)[N], int C, const LineScales& c) {
    return win_d1(w, C, c);
  }
  // first derivative kept for composition (D_x, D_y fields)
  template <int N>
  static __device__ __forceinline__ double d1_field(const double (&w)[N], int C, const LineScales& c) {
    return win_d1(w, C, c);
  }
  template <int N>
  static __device__ __forceinline__ D d2(const double (&w)[N], int C, const LineScales& c) {
    return win_d2(w, C, c);
  }
  template <int N>
  static __device__ __forceinline__ double ko(const double (&w)[N], int C, const LineScales& c) {
    return win_ko(w, C, c);
  }
  // upwind advective row `row` (adv_row_id) in the reference's order, each op rounded
  template <int N>
  static __device__ __forceinline__ D adv(const double (&w)[N], int C, int row, const LineScales& c) {
    double a;
    switch (row) {
      case 0:
        a = __dmul_rn(-3.0, w[C - 1]); a = mad_rn(a, -10.0, w[C]); a = mad_rn(a, 18.0, w[C + 1]);
        a = mad_rn(a, -6.0, w[C + 2]); a = mad_rn(a, 1.0, w[C + 3]);
        return __dmul_rn(a, c.d1_b);
      case 1:
        a = __dmul_rn(-1.0, w[C - 3]); a = mad_rn(a, 6.0, w[C - 2]); a = mad_rn(a, -18.0, w[C - 1]);
        a = mad_rn(a, 10.0, w[C]); a = mad_rn(a, 3.0, w[C + 1]);
        return __dmul_rn(a, c.d1_b);
      case 2:
        a = __dmul_rn(-3.0, w[C]); a = mad_rn(a, 4.0, w[C + 1]); a = mad_rn(a, -1.0, w[C + 2]);
        return __dmul_rn(a, c.adv_b2);
      case 3:
        a = __dmul_rn(-1.0, w[C - 1]); a = mad_rn(a, 1.0, w[C + 1]);
        return __dmul_rn(a, c.adv_b2);
      default:
        a = __dmul_rn(1.0, w[C - 2]); a = mad_rn(a, -4.0, w[C - 1]); a = mad_rn(a, 3.0, w[C]);
        return __dmul_rn(a, c.adv_b2);
    }
  }
};

struct SplitRows {
  using D = float;
  // the weighted sum of the FP64 differences is formed in FP64 and rounded once to the
  // FP32 of the slot: one rounding instead of four, and no conversion per difference
  template <typename T, int N>
  static __device__ __forceinline__ D d1(const T (&w)[N], int C, const LineScales& c) {
    const double a1 = (double)w[C + 1] - (double)w[C - 1];
    const double a2 = (double)w[C + 2] - (double)w[C - 2];
    const double a3 = (double)w[C + 3] - (double)w[C - 3];
    return (float)(fma(45.0, a1, fma(-9.0, a2, a3)) * c.d1_c);
  }
  // D_x / D_y fields that feed the mixed derivatives stay FP64: differencing
  // FP32-rounded first derivatives would cancel their leading digits
  template <int N>
  static __device__ __forceinline__ double d1_field(const double (&w)[N], int C, const LineScales& c) {
    const double a1 = w[C + 1] - w[C - 1];
    const double a2 = w[C + 2] - w[C - 2];
    const double a3 = w[C + 3] - w[C - 3];
    return fma(45.0, a1, fma(-9.0, a2, a3)) * c.d1_c;
  }
  template <int N>
  static __device__ __forceinline__ D d2(const double (&w)[N], int C, const LineScales& c) {
    const double u2 = 2.0 * w[C];
    const double s1 = (w[C + 1] + w[C - 1]) - u2;
    const double s2 = (w[C + 2] + w[C - 2]) - u2;
    const double s3 = (w[C + 3] + w[C - 3]) - u2;
    return (float)(fma(270.0, s1, fma(-27.0, s2, 2.0 * s3)) * c.d2_c);
  }
  template <int N>
  static __device__ __forceinline__ double ko(const double (&w)[N], int C, const LineScales& c) {
    const double u2 = 2.0 * w[C];
    const double s1 = (w[C + 1] + w[C - 1]) - u2;
    const double s2 = (w[C + 2] + w[C - 2]) - u2;
    const double s3 = (w[C + 3] + w[C - 3]) - u2;
    return c.ko_c * fma(-15.0, s1, fma(6.0, s2, -s3));
  }
  // upwind advective rows: the weights sum to zero, so the row is a weighted sum of FP64
  // differences from the centre value, summed in FP32
  template <int N>
  static __device__ __forceinline__ D adv(const double (&w)[N], int C, int row, const LineScales& c) {
    auto dd = [&](int k) { return (float)(w[C + k] - w[C]); };
    switch (row) {
      case 0:
        return fmaf(-3.0f, dd(-1), fmaf(18.0f, dd(1), fmaf(-6.0f, dd(2), dd(3)))) * (float)c.d1_b;
      case 1:
        return fmaf(6.0f, dd(-2), fmaf(-18.0f, dd(-1), fmaf(3.0f, dd(1), -dd(-3)))) * (float)c.d1_b;
      case 2:
        return fmaf(4.0f, dd(1), -dd(2)) * (float)c.adv_b2;
      case 3:
        return (float)(w[C + 1] - w[C - 1]) * (float)c.adv_b2;
      default:
        return fmaf(-4.0f, dd(-1), dd(-2)) * (float)c.adv_b2;
    }
  }
};

// Closure rows (rare: next to flagged faces) on shared memory, evaluated exactly
// in FP64; float values (MIXED-mode D_x/D_y fields) are widened first.
template <typename T>
static __device__ __noinline__ double cl_d1(const T* p, int s, int pos, int n, bool lo, bool hi,
                                            const LineScales& c) {
  double v[9];  // values at pos-4 .. pos+4 that lie inside [0, n)
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int at = pos + k - 4;
    v[k] = (at >= 0 && at < n) ? (double)p[(k - 4) * s] : 0.0;
  }
  return line_d1(v + 4, 1, pos, n, lo, hi, c);
}
template <typename T>
static __device__ __noinline__ double cl_d2(const T* p, int s, int pos, int n, bool lo, bool hi,
                                            const LineScales& c) {
  double v[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int at = pos + k - 4;
    v[k] = (at >= 0 && at < n) ? (double)p[(k - 4) * s] : 0.0;
  }
  return line_d2(v + 4, 1, pos, n, lo, hi, c);
}
template <typename T>
static __device__ __noinline__ double cl_ko(const T* p, int s, int pos, int n, bool lo, bool hi,
                                            const LineScales& c) {
  double v[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int at = pos + k - 4;
    v[k] = (at >= 0 && at < n) ? (double)p[(k - 4) * s] : 0.0;
  }
  return line_ko(v + 4, 1, pos, n, lo, hi, c);
}

template <typename ST>
struct RowsFor { using type = ExactRows; };
template <>
struct RowsFor<float> { using type = SplitRows; };

// One (column tile, variable) work item; DD: the variable has second derivatives;
// ADV: also the upwind advective derivatives (slots kNumDerivs + 3v + axis, upwinded
// by the sign of the matching shift component at the point); CL: some point of the
// item takes a closure row (tile_has_closure) -- without, the closure branches and
// the face cases of the upwind rows compile away.
//
// Scratch point of output (tile column tx, ty; plane zo of the slab): lp = col_base +
// tx + row_stride * ty + plane_pts * zo -- the unit's compact numbering on the two-pass
// path, the tile's own 16x8-per-plane numbering inside a ring slot on the single-pass path.
struct ScratchMap {
  int32_t col_base, row_stride, plane_pts;
};

template <typename ST, bool DD, bool ADV = false, bool CL = true, int TY = kTileY>
__device__ __forceinline__ void derive_item(const DerivArgs& a, const UnitDev& un, const TileDev& t,
                                            const ScratchMap sm, const int v, double* s_plane,
                                            void* s_dxp_raw, double* s_kq, LineScales* s_sc) {
  using Rows = typename RowsFor<ST>::type;
  using SH = TileShape<TY>;
  constexpr int NS = ADV ? kNumDerivs + 3 * kNumVars : kNumDerivs;  // slots per point
  double* s_dxp = static_cast<double*>(s_dxp_raw);
  const BlockDev& B = a.blocks[un.block];
  const int nx = B.sz[0], ny = B.sz[1], nz = B.sz[2];
  const int i0 = 3 + t.i0, j0 = 3 + t.j0, k0 = 3 + un.k0;
  const int ex = t.ex, ey = t.ey, ez = un.nz;
  const int ox = i0 - kHalo, oy = j0 - kHalo;  // plane origin (padded coords)
  const int xlo = max(0, ox), xhi = min(nx, i0 + ex + kHalo);
  const int ylo = max(0, oy), yhi = min(ny, j0 + ey + kHalo);
  const uint32_t bf = B.bflag;
  const bool lox = CL && (bf & 1u), hix = CL && (bf & 2u), loy = CL && (bf & 4u),
             hiy = CL && (bf & 8u), loz = CL && (bf & 16u), hiz = CL && (bf & 32u);
  if (threadIdx.x < 3) s_sc[threadIdx.x] = make_line_scales(B.h[threadIdx.x]);

  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const bool active = tx < ex && ty < ey;
  const int gi = i0 + tx, gj = j0 + ty;
  // chunk-relative scratch offsets fit in 32 bits (NS * cap < 2^31)
  const int plane_pts = sm.plane_pts;
  const int lp_col = sm.col_base + tx + sm.row_stride * ty;  // + plane_pts * (z - k0)
  // z reach of the item's rows: closure rows reach 4 planes, centred rows 3
  constexpr int H = CL ? kHalo : 3;
  constexpr int QD = 2 * H + 1;
  const int zs = max(0, k0 - H);
  const int zend = k0 + ez + H;  // exclusive
  const int zload = min(nz, zend);   // planes beyond are never loaded
  const bool clx = closure_row(gi, nx, lox, hix), cly = closure_row(gj, ny, loy, hiy);

  // This thread's share of a plane copy (fixed for the whole item): column sbx of
  // the 32-wide staging grid (24 columns used), every (warps per CTA)-th row of the
  // plane from its warp's index on.
  const int sbx = threadIdx.x & 31, sby0 = threadIdx.x >> 5;
  int st_soff[SH::kStageRows], st_goff[SH::kStageRows];
  bool st_ok[SH::kStageRows];
#pragma unroll
  for (int r = 0; r < SH::kStageRows; ++r) {
    const int by = sby0 + SH::kWarps * r, pi = ox + sbx, pj = oy + by;
    st_ok[r] = sbx < kPlaneW && pi >= xlo && pi < xhi && pj >= ylo && pj < yhi;
    st_soff[r] = by * kPlaneW + sbx;
    st_goff[r] = pi + nx * pj;
  }
  // and of the y-halo D_x rows: column dxx, rows dyy0, dyy0 + TY, ...
  const int dxx = threadIdx.x & 15, dyy0 = threadIdx.x >> 4;
  const int dpi = i0 + dxx;
  const bool dcl = closure_row(dpi, nx, lox, hix);
  bool dx_ok[SH::kDxPerThread];
#pragma unroll
  for (int r = 0; r < SH::kDxPerThread; ++r) {
    const int yy = dyy0 + TY * r, pj = oy + yy;
    dx_ok[r] = yy < SH::kDxRows && dxx < ex && pj >= ylo && pj < yhi;
  }
  const int64_t plane_elems = (int64_t)nx * ny;

  const int q = DD ? dd_index(v) : -1;
  const double* __restrict__ f = a.u[v] + B.offset;
  // The item's scratch columns: slot s of point lp sits at (lp / 32) * 32 NS + s * 32 +
  // lp % 32 (scr_index), so per output point one offset serves every slot of the
  // variable, each store adding a constant.
  ST* const sd_first = static_cast<ST*>(a.dscr) + (3 * v) * 32;                        // D_x, D_y, D_z
  ST* const sd_second = static_cast<ST*>(a.dscr) + (72 + 6 * (DD ? q : 0)) * 32;       // the 6 second
  ST* const sd_adv = static_cast<ST*>(a.dscr) + (kNumDerivs + 3 * v) * 32;              // upwind mode
  ST* const sk = static_cast<ST*>(a.koscr) + v * 32;                                     // KO sum
  auto col = [](int lp) { return (lp >> 5) * (NS * 32) + (lp & 31); };
  auto kcol = [](int lp) { return (lp >> 5) * (kNumVars * 32) + (lp & 31); };
  double qu[QD], qx[QD], qy[QD];  // planes zi-2H .. zi of u, D_x u, D_y u (D_x/D_y: DD only)
  int kslot = 0;  // ring slot of plane zi's (ko_x + ko_y) in s_kq (H + 1 planes deep)
#pragma unroll
  for (int k = 0; k < QD; ++k) qu[k] = qx[k] = qy[k] = 0.0;

  // stage plane zi into buffer b (one commit group; empty past the last needed plane);
  // predicated copies, no branches
  auto stage = [&](int zi, int b) {
    const double* fp = f + plane_elems * zi;
    const bool in = zi < zload;
#pragma unroll
    for (int r = 0; r < SH::kStageRows; ++r)
      cp_async8_if(s_plane + b * SH::kPlane + st_soff[r], fp + st_goff[r], in && st_ok[r]);
    cp_async_commit();
  };

  // Four plane buffers: plane zi+3 streams into the buffer plane zi-1 used, which
  // every thread has finished with once it passes the barrier of step zi.  For DD
  // variables step zi also differentiates plane zi+1 along x on the y-halo rows
  // (into the other of two D_x buffers), so one barrier per step orders both the
  // plane copies and the D_x rows.
  const LineScales& cx = s_sc[0];
  const LineScales& cy = s_sc[1];
  auto dx_rows = [&](int zp, const double* P, double* dst) {
    if (zp < zload) {
#pragma unroll
      for (int r = 0; r < SH::kDxPerThread; ++r) {
        if (dx_ok[r]) {
          const int yy = dyy0 + TY * r;
          const double* p = P + yy * kPlaneW + dxx + kHalo;
          double w[7];
#pragma unroll
          for (int k = 0; k < 7; ++k) w[k] = p[k - 3];
          dst[yy * kTileX + dxx] = dcl ? cl_d1(p, 1, dpi, nx, lox, hix, cx) : Rows::d1_field(w, 3, cx);
        }
      }
    }
  };
  stage(zs, 0);
  stage(zs + 1, 1);
  stage(zs + 2, 2);
  if (DD) {
    cp_async_wait<2>();
    __syncthreads();  // plane zs (and the line scales) visible to every thread
    dx_rows(zs, s_plane, s_dxp);
  }
  for (int zi = zs, b = 0; zi < zend; ++zi, b = (b + 1) & 3) {
    cp_async_wait<1>();
    __syncthreads();
    stage(zi + 3, (b + 3) & 3);
    const double* P = s_plane + b * SH::kPlane;
    const double* Dxp = s_dxp + ((zi - zs) & 1) * (SH::kDxRows * kTileX);
    const bool in_block = zi < nz;
    const bool out_plane = zi >= k0 && zi < k0 + ez;
    if (DD) dx_rows(zi + 1, s_plane + ((b + 1) & 3) * SH::kPlane, s_dxp + ((zi + 1 - zs) & 1) * (SH::kDxRows * kTileX));

    double dx = 0.0, dy = 0.0, kxy = 0.0, u0 = 0.0;
    if (active && in_block) {
      const double* pc = P + (ty + kHalo) * kPlaneW + (tx + kHalo);
      u0 = *pc;
    }
    // halo planes only feed the z queues: u for every kind, D_x u and D_y u for DD
    if (active && in_block && (DD || out_plane)) {
      const double* pc = P + (ty + kHalo) * kPlaneW + (tx + kHalo);
      double wx[7], wy[7];
#pragma unroll
      for (int k = 0; k < 7; ++k) {
        wx[k] = pc[k - 3];
        wy[k] = pc[(k - 3) * kPlaneW];
      }
      dx = DD ? Dxp[(ty + kHalo) * kTileX + tx]
                  : (clx ? cl_d1(pc, 1, gi, nx, lox, hix, cx) : Rows::d1_field(wx, 3, cx));
      dy = cly ? cl_d1(pc, kPlaneW, gj, ny, loy, hiy, cy) : Rows::d1_field(wy, 3, cy);
      if (out_plane) {
        const int lp = lp_col + plane_pts * (zi - k0);
        const double kx = clx ? cl_ko(pc, 1, gi, nx, lox, hix, cx) : Rows::ko(wx, 3, cx);
        const double ky = cly ? cl_ko(pc, kPlaneW, gj, ny, loy, hiy, cy) : Rows::ko(wy, 3, cy);
        s_kq[kslot * SH::kThreads + threadIdx.x] = __dadd_rn(kx, ky);
        const int c = col(lp);
        sd_first[c] = (ST)dx;
        sd_first[c + 32] = (ST)dy;
        if (DD) {
          sd_second[c + 0 * 32] = (ST)(clx ? cl_d2(pc, 1, gi, nx, lox, hix, cx) : (double)Rows::d2(wx, 3, cx));
          sd_second[c + 3 * 32] = (ST)(cly ? cl_d2(pc, kPlaneW, gj, ny, loy, hiy, cy) : (double)Rows::d2(wy, 3, cy));
          const double* pd = Dxp + (ty + kHalo) * kTileX + tx;
          double wd[7];
#pragma unroll
          for (int k = 0; k < 7; ++k) wd[k] = pd[(k - 3) * kTileX];
          sd_second[c + 1 * 32] = (ST)(cly ? cl_d1(pd, kTileX, gj, ny, loy, hiy, cy) : (double)Rows::d1(wd, 3, cy));
        }
        if constexpr (ADV) {
          // deriv42adv_x / _y (derivs.cpp:495-775) with beta0 / beta1 at the point
          const int64_t pe = (int64_t)B.offset + gi + (int64_t)nx * gj + plane_elems * zi;
          const bool upx = __ldg(a.u[6] + pe) > 0.0, upy = __ldg(a.u[7] + pe) > 0.0;
          sd_adv[c] = (ST)(double)Rows::adv(wx, 3, adv_row_id(gi, nx, lox, hix, upx), cx);
          sd_adv[c + 32] = (ST)(double)Rows::adv(wy, 3, adv_row_id(gj, ny, loy, hiy, upy), cy);
        }
      }
    }
    q_push(qu, u0);
    if (DD) {
      q_push(qx, dx);
      q_push(qy, dy);
    }
    // (ko_x + ko_y) of plane zi - H, written H steps ago into slot kslot - H (mod H + 1)
    const int kold = kslot == H ? 0 : kslot + 1;
    kxy = s_kq[kold * SH::kThreads + threadIdx.x];
    kslot = kold;

    // z derivatives of plane zo = zi - H, whose +-H neighbourhood is now queued
    const int zo = zi - H;
    if (active && zo >= k0 && zo < k0 + ez) {
      const LineScales& cz = s_sc[2];
      const int zc = CL ? z_case(zo, nz, loz, hiz) : -1;
      const int lp = lp_col + plane_pts * (zo - k0);
      const int c = col(lp);
      sd_first[c + 2 * 32] = (ST)zrow_d1<CL, Rows>(qu, zc, cz);
      // rhs.cpp:332-369 sums (ko_x + ko_y) + ko_z
      // summed in FP64, stored like the slots (FP32 in MIXED: the term enters the output
      // scaled by sigma, far below the output's own scale)
      sk[kcol(lp)] = (ST)__dadd_rn(kxy, zrow_ko<CL, Rows>(qu, zc, cz));
      if (DD) {
        sd_second[c + 5 * 32] = (ST)zrow_d2<CL, Rows>(qu, zc, cz);
        sd_second[c + 2 * 32] = (ST)zrow_d1<CL, Rows>(qx, zc, cz);
        sd_second[c + 4 * 32] = (ST)zrow_d1<CL, Rows>(qy, zc, cz);
      }
      if constexpr (ADV) {
        // deriv42adv_z (derivs.cpp:776-900) with beta2 at the point
        const int64_t pe = (int64_t)B.offset + gi + (int64_t)nx * gj + plane_elems * zo;
        const bool upz = __ldg(a.u[8] + pe) > 0.0;
        sd_adv[c + 2 * 32] = (ST)(double)Rows::adv(qu, H, adv_row_id(zo, nz, loz, hiz, upz), cz);
      }
    }
  }
  cp_async_wait<0>();
}

// The same item with two output points per thread: a 16x16 tile in a CTA of 128
// threads, thread (tx, tq) owning rows 2tq and 2tq+1.  The two points share one y
// window (8 plane values instead of 14) and one D_x y window, and the per-step loop,
// barrier, plane copy and predicate work is spread over two points; each point keeps
// its own z queues.  Centred advection only (no upwind rows).
template <typename ST, bool DD, bool CL = true>
__device__ __forceinline__ void derive_item_pair(const DerivArgs& a, const UnitDev& un, const TileDev& t,
                                                 const ScratchMap sm, const int v, double* s_plane,
                                                 void* s_dxp_raw, double* s_kq, LineScales* s_sc) {
  using Rows = typename RowsFor<ST>::type;
  constexpr int NS = kNumDerivs;
  constexpr int NT = 128, TR = 16, WARPS = NT / 32;
  constexpr int PH = TR + 2 * kHalo, PLANE = kPlaneW * PH;  // 24 x 24 staged plane
  constexpr int SROWS = PH / WARPS;                          // plane rows per thread
  constexpr int DXR = TR + 2 * kHalo, DXT = DXR / (NT / kTileX);  // D_x halo rows: 24, 3 per thread
  static_assert(SROWS * WARPS == PH && DXT * (NT / kTileX) == DXR, "pair tile geometry");
  double* s_dxp = static_cast<double*>(s_dxp_raw);
  const BlockDev& B = a.blocks[un.block];
  const int nx = B.sz[0], ny = B.sz[1], nz = B.sz[2];
  const int i0 = 3 + t.i0, j0 = 3 + t.j0, k0 = 3 + un.k0;
  const int ex = t.ex, ey = t.ey, ez = un.nz;
  const int ox = i0 - kHalo, oy = j0 - kHalo;
  const int xlo = max(0, ox), xhi = min(nx, i0 + ex + kHalo);
  const int ylo = max(0, oy), yhi = min(ny, j0 + ey + kHalo);
  const uint32_t bf = B.bflag;
  const bool lox = CL && (bf & 1u), hix = CL && (bf & 2u), loy = CL && (bf & 4u),
             hiy = CL && (bf & 8u), loz = CL && (bf & 16u), hiz = CL && (bf & 32u);
  if (threadIdx.x < 3) s_sc[threadIdx.x] = make_line_scales(B.h[threadIdx.x]);

  const int tx = threadIdx.x & 15, tq = threadIdx.x >> 4, ty0 = 2 * tq;
  const int gi = i0 + tx;
  const bool clx = closure_row(gi, nx, lox, hix);
  bool active[2], cly[2];
  int gj[2], lp_col[2];
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    active[p] = tx < ex && ty0 + p < ey;
    gj[p] = j0 + ty0 + p;
    cly[p] = closure_row(gj[p], ny, loy, hiy);
    lp_col[p] = sm.col_base + tx + sm.row_stride * (ty0 + p);
  }
  const bool any = active[0] || active[1];
  const int plane_pts = sm.plane_pts;
  constexpr int H = CL ? kHalo : 3;
  constexpr int QD = 2 * H + 1;
  const int zs = max(0, k0 - H);
  const int zend = k0 + ez + H;
  const int zload = min(nz, zend);

  const int sbx = threadIdx.x & 31, sby0 = threadIdx.x >> 5;
  int st_soff[SROWS], st_goff[SROWS];
  bool st_ok[SROWS];
#pragma unroll
  for (int r = 0; r < SROWS; ++r) {
    const int by = sby0 + WARPS * r, pi = ox + sbx, pj = oy + by;
    st_ok[r] = sbx < kPlaneW && pi >= xlo && pi < xhi && pj >= ylo && pj < yhi;
    st_soff[r] = by * kPlaneW + sbx;
    st_goff[r] = pi + nx * pj;
  }
  const int dxx = threadIdx.x & 15, dyy0 = threadIdx.x >> 4;
  const int dpi = i0 + dxx;
  const bool dcl = closure_row(dpi, nx, lox, hix);
  bool dx_ok[DXT];
#pragma unroll
  for (int r = 0; r < DXT; ++r) {
    const int yy = dyy0 + (NT / kTileX) * r, pj = oy + yy;
    dx_ok[r] = yy < DXR && dxx < ex && pj >= ylo && pj < yhi;
  }
  const int64_t plane_elems = (int64_t)nx * ny;

  const int q = DD ? dd_index(v) : -1;
  const double* __restrict__ f = a.u[v] + B.offset;
  ST* const sd_first = static_cast<ST*>(a.dscr) + (3 * v) * 32;
  ST* const sd_second = static_cast<ST*>(a.dscr) + (72 + 6 * (DD ? q : 0)) * 32;
  ST* const sk = static_cast<ST*>(a.koscr) + v * 32;
  auto col = [](int lp) { return (lp >> 5) * (NS * 32) + (lp & 31); };
  auto kcol = [](int lp) { return (lp >> 5) * (kNumVars * 32) + (lp & 31); };
  double qu[2][QD], qx[2][QD], qy[2][QD];
  int kslot = 0;
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int k = 0; k < QD; ++k) qu[p][k] = qx[p][k] = qy[p][k] = 0.0;

  auto stage = [&](int zi, int b) {
    const double* fp = f + plane_elems * zi;
    const bool in = zi < zload;
#pragma unroll
    for (int r = 0; r < SROWS; ++r) cp_async8_if(s_plane + b * PLANE + st_soff[r], fp + st_goff[r], in && st_ok[r]);
    cp_async_commit();
  };
  const LineScales& cx = s_sc[0];
  const LineScales& cy = s_sc[1];
  auto dx_rows = [&](int zp, const double* P, double* dst) {
    if (zp < zload) {
#pragma unroll
      for (int r = 0; r < DXT; ++r) {
        if (dx_ok[r]) {
          const int yy = dyy0 + (NT / kTileX) * r;
          const double* pr = P + yy * kPlaneW + dxx + kHalo;
          double w[7];
#pragma unroll
          for (int k = 0; k < 7; ++k) w[k] = pr[k - 3];
          dst[yy * kTileX + dxx] = dcl ? cl_d1(pr, 1, dpi, nx, lox, hix, cx) : Rows::d1_field(w, 3, cx);
        }
      }
    }
  };
  stage(zs, 0);
  stage(zs + 1, 1);
  stage(zs + 2, 2);
  if (DD) {
    cp_async_wait<2>();
    __syncthreads();
    dx_rows(zs, s_plane, s_dxp);
  }
  for (int zi = zs, b = 0; zi < zend; ++zi, b = (b + 1) & 3) {
    cp_async_wait<1>();
    __syncthreads();
    stage(zi + 3, (b + 3) & 3);
    const double* P = s_plane + b * PLANE;
    const double* Dxp = s_dxp + ((zi - zs) & 1) * (DXR * kTileX);
    const bool in_block = zi < nz;
    const bool out_plane = zi >= k0 && zi < k0 + ez;
    if (DD) dx_rows(zi + 1, s_plane + ((b + 1) & 3) * PLANE, s_dxp + ((zi + 1 - zs) & 1) * (DXR * kTileX));

    double u0[2] = {0.0, 0.0}, dx[2] = {0.0, 0.0}, dy[2] = {0.0, 0.0};
    const double* pc0 = P + (ty0 + kHalo) * kPlaneW + (tx + kHalo);
    if (any && in_block) {
      u0[0] = active[0] ? pc0[0] : 0.0;
      u0[1] = active[1] ? pc0[kPlaneW] : 0.0;
    }
    if (any && in_block && (DD || out_plane)) {
      double wy8[8];  // rows ty0-3 .. ty0+4 of column tx: the y windows of both points
#pragma unroll
      for (int k = 0; k < 8; ++k) wy8[k] = pc0[(k - 3) * kPlaneW];
      double wd8[8];  // the same rows of D_x (DD)
      if (DD) {
        const double* pd0 = Dxp + (ty0 + kHalo) * kTileX + tx;
#pragma unroll
        for (int k = 0; k < 8; ++k) wd8[k] = pd0[(k - 3) * kTileX];
      }
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        if (!active[p]) continue;
        const double* pc = pc0 + p * kPlaneW;
        double wx[7], wy[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) {
          wx[k] = pc[k - 3];
          wy[k] = wy8[k + p];
        }
        dx[p] = DD ? wd8[3 + p] : (clx ? cl_d1(pc, 1, gi, nx, lox, hix, cx) : Rows::d1_field(wx, 3, cx));
        dy[p] = cly[p] ? cl_d1(pc, kPlaneW, gj[p], ny, loy, hiy, cy) : Rows::d1_field(wy, 3, cy);
        if (out_plane) {
          const int lp = lp_col[p] + plane_pts * (zi - k0);
          const double kx = clx ? cl_ko(pc, 1, gi, nx, lox, hix, cx) : Rows::ko(wx, 3, cx);
          const double ky = cly[p] ? cl_ko(pc, kPlaneW, gj[p], ny, loy, hiy, cy) : Rows::ko(wy, 3, cy);
          s_kq[(kslot * NT + threadIdx.x) * 2 + p] = __dadd_rn(kx, ky);
          const int c = col(lp);
          sd_first[c] = (ST)dx[p];
          sd_first[c + 32] = (ST)dy[p];
          if (DD) {
            sd_second[c + 0 * 32] = (ST)(clx ? cl_d2(pc, 1, gi, nx, lox, hix, cx) : (double)Rows::d2(wx, 3, cx));
            sd_second[c + 3 * 32] = (ST)(cly[p] ? cl_d2(pc, kPlaneW, gj[p], ny, loy, hiy, cy) : (double)Rows::d2(wy, 3, cy));
            double wd[7];
#pragma unroll
            for (int k = 0; k < 7; ++k) wd[k] = wd8[k + p];
            const double* pd = Dxp + (ty0 + p + kHalo) * kTileX + tx;
            sd_second[c + 1 * 32] = (ST)(cly[p] ? cl_d1(pd, kTileX, gj[p], ny, loy, hiy, cy) : (double)Rows::d1(wd, 3, cy));
          }
        }
      }
    }
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      q_push(qu[p], u0[p]);
      if (DD) {
        q_push(qx[p], dx[p]);
        q_push(qy[p], dy[p]);
      }
    }
    const int kold = kslot == H ? 0 : kslot + 1;
    double kxy[2];
#pragma unroll
    for (int p = 0; p < 2; ++p) kxy[p] = s_kq[(kold * NT + threadIdx.x) * 2 + p];
    kslot = kold;

    const int zo = zi - H;
    if (zo >= k0 && zo < k0 + ez) {
      const LineScales& cz = s_sc[2];
      const int zc = CL ? z_case(zo, nz, loz, hiz) : -1;
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        if (!active[p]) continue;
        const int lp = lp_col[p] + plane_pts * (zo - k0);
        const int c = col(lp);
        sd_first[c + 2 * 32] = (ST)zrow_d1<CL, Rows>(qu[p], zc, cz);
        sk[kcol(lp)] = (ST)__dadd_rn(kxy[p], zrow_ko<CL, Rows>(qu[p], zc, cz));
        if (DD) {
          sd_second[c + 5 * 32] = (ST)zrow_d2<CL, Rows>(qu[p], zc, cz);
          sd_second[c + 2 * 32] = (ST)zrow_d1<CL, Rows>(qx[p], zc, cz);
          sd_second[c + 4 * 32] = (ST)zrow_d1<CL, Rows>(qy[p], zc, cz);
        }
      }
    }
  }
  cp_async_wait<0>();
}

// Two-pass path: item (tile t of a unit, variable v) with the unit's compact scratch
// numbering.
template <typename ST, bool DD, bool ADV = false, bool CL = true, int TY = kTileY>
__device__ __forceinline__ void derive_tile(const DerivArgs& a, const TileDev t, const int v,
                                            double* s_plane, void* s_dxp_raw,
                                            double* s_kq, LineScales* s_sc) {
  const UnitDev un = a.units[t.unit];
  const int I0 = a.blocks[un.block].sz[0] - 6, I1 = a.blocks[un.block].sz[1] - 6;
  const ScratchMap sm{(int)un.sbase + t.i0 + I0 * t.j0, I0, I0 * I1};
  derive_item<ST, DD, ADV, CL, TY>(a, un, t, sm, v, s_plane, s_dxp_raw, s_kq, s_sc);
}

// True when some output point of the item lies within three points of a flagged
// face (closure_row on the tile's x and y ranges or the slab's z range).
__device__ __forceinline__ bool item_has_closure(const BlockDev& B, const UnitDev& un, const TileDev& t) {
  const uint32_t bf = B.bflag;
  auto near = [](int p0, int e, int n, bool lo, bool hi) { return (lo && p0 < 6) || (hi && p0 + e - 1 >= n - 6); };
  return near(3 + t.i0, t.ex, B.sz[0], bf & 1u, bf & 2u) || near(3 + t.j0, t.ey, B.sz[1], bf & 4u, bf & 8u) ||
         near(3 + un.k0, un.nz, B.sz[2], bf & 16u, bf & 32u);
}
__device__ __forceinline__ bool tile_has_closure(const DerivArgs& a, const TileDev& t) {
  const UnitDev un = a.units[t.unit];
  return item_has_closure(a.blocks[un.block], un, t);
}

// Persistent derivative kernel: the grid holds as many CTAs as fit on the GPU at
// once, and each CTA takes the next (tile, variable) item of the chunk from a
// device counter (the planner lists a chunk's tiles longest first); an item is
// one variable streamed through one column tile, so the launch ends with a short
// tail whatever the mix of block sizes.
template <typename ST>
__global__ void __launch_bounds__(kDerivThreads, 512 / kDerivThreads)
bssn_derivs_kernel(const __grid_constant__ DerivArgs a) {
  __shared__ double s_plane[4][kPlane];
  __shared__ double s_dxp[2 * kDxRows * kTileX];
  __shared__ double s_kq[(kHalo + 1) * kDerivThreads];
  __shared__ LineScales s_sc[3];
  __shared__ int s_item;
  for (;;) {
    __syncthreads();  // the previous item is finished with every shared array
    if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= a.tile_count * kNumVars) break;
    // items run tile-major: the longest tiles (listed first) are all taken first
    const TileDev t = a.tiles[a.tile_base + item / kNumVars];
    const int v = item % kNumVars;
    const bool cl = tile_has_closure(a, t);
    if (dd_index(v) >= 0) {
      if (cl)
        derive_tile<ST, true, false, true>(a, t, v, &s_plane[0][0], s_dxp, s_kq, s_sc);
      else
        derive_tile<ST, true, false, false>(a, t, v, &s_plane[0][0], s_dxp, s_kq, s_sc);
    } else {
      if (cl)
        derive_tile<ST, false, false, true>(a, t, v, &s_plane[0][0], s_dxp, s_kq, s_sc);
      else
        derive_tile<ST, false, false, false>(a, t, v, &s_plane[0][0], s_dxp, s_kq, s_sc);
    }
  }
}

constexpr size_t kDerivSmemBytes = 0;  // all shared memory is static

// The same items split by kind into two persistent kernels, one over the 11
// variables with second derivatives and one over the 13 without: the latter needs
// fewer registers than 128, so it runs more warps per SM (measured on the batch, with
// 16x16 tiles, 80 registers against 128: derivatives 70.0 -> 62.8 ms MIXED, 76.9 ->
// 71.0 ms FP64); it now runs 5 CTAs per SM at up to 96 registers without spills (6 at
// 80: MIXED the same, FP64 1 % slower).  The CTA is a 16x8 tile of 4 warps, so each
// per-plane barrier waits on 4 warps (16x16 tiles of 8 warps: 48.8 / 64.0 ms against
// 47.5 / 63.6 ms, despite the larger halo share).  Plans launch
// these; the allocation-free entry point keeps the combined kernel above.
__device__ __forceinline__ int kind_var(bool dd, int i) {
  constexpr int kDD[11] = {0, 1, 6, 7, 8, 12, 13, 14, 15, 16, 17};  // alpha chi beta gt
  constexpr int kND[13] = {2, 3, 4, 5, 9, 10, 11, 18, 19, 20, 21, 22, 23};  // K Gt B At
  return dd ? kDD[i] : kND[i];
}
constexpr int kKindVars[2] = {13, 11};        // [DD]
// Launch-bound occupancy of a kind kernel (its registers-per-thread split): the CTAs
// per SM for 16x8 tiles -- 5 for the first-derivative kind (96 registers; the upwind
// first-derivative kind keeps 6: 5 measured 4 % slower there), 4 for the second-
// derivative kind (128) -- scaled to keep the warps per SM for other tile heights;
// variant REGV 1 asks for one more CTA per SM (fewer registers), 2 for one fewer.
constexpr int kind_ctas_per_sm(bool dd, bool adv, int ty = kTileY, int regv = 0) {
  const int base = (dd ? 512 : (adv ? 768 : 640)) / (kTileX * ty);
  return regv == 1 ? base + 1 : (regv == 2 ? (base > 1 ? base - 1 : 1) : base);
}

template <typename ST, bool DD, bool ADV = false, int TY = kTileY, int REGV = 0>
__global__ void __launch_bounds__(TileShape<TY>::kThreads, kind_ctas_per_sm(DD, ADV, TY, REGV))
bssn_derivs_kind_kernel(const __grid_constant__ DerivArgs a) {
  using SH = TileShape<TY>;
  constexpr int NV = kKindVars[DD];
  __shared__ double s_plane[4 * SH::kPlane];
  __shared__ double s_dxp[DD ? 2 * SH::kDxRows * kTileX : 1];
  __shared__ double s_kq[(kHalo + 1) * SH::kThreads];
  __shared__ LineScales s_sc[3];
  __shared__ int s_item;
  for (;;) {
    __syncthreads();  // the previous item is finished with every shared array
    if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= a.tile_count * NV) break;
    const TileDev t = a.tiles[a.tile_base + item / NV];
    if (tile_has_closure(a, t))
      derive_tile<ST, DD, ADV, true, TY>(a, t, kind_var(DD, item % NV), s_plane, s_dxp, s_kq, s_sc);
    else
      derive_tile<ST, DD, ADV, false, TY>(a, t, kind_var(DD, item % NV), s_plane, s_dxp, s_kq, s_sc);
  }
}

// The derivative kinds with two output points per thread (derive_item_pair) on 16x16
// tiles in CTAs of 128 threads; CTAs per SM: 3 without second derivatives, 2 with.
constexpr int pair_ctas_per_sm(bool dd) { return dd ? 2 : 3; }

template <typename ST, bool DD>
__global__ void __launch_bounds__(128, pair_ctas_per_sm(DD))
bssn_derivs_pair_kernel(const __grid_constant__ DerivArgs a) {
  constexpr int NV = kKindVars[DD];
  constexpr int PLANE = kPlaneW * (16 + 2 * kHalo);
  __shared__ double s_plane[4 * PLANE];
  __shared__ double s_dxp[DD ? 2 * (16 + 2 * kHalo) * kTileX : 1];
  __shared__ double s_kq[(kHalo + 1) * 128 * 2];
  __shared__ LineScales s_sc[3];
  __shared__ int s_item;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= a.tile_count * NV) break;
    const TileDev t = a.tiles[a.tile_base + item / NV];
    const UnitDev un = a.units[t.unit];
    const int I0 = a.blocks[un.block].sz[0] - 6, I1 = a.blocks[un.block].sz[1] - 6;
    const ScratchMap sm{(int)un.sbase + t.i0 + I0 * t.j0, I0, I0 * I1};
    const int v = kind_var(DD, item % NV);
    if (item_has_closure(a.blocks[un.block], un, t))
      derive_item_pair<ST, DD, true>(a, un, t, sm, v, s_plane, s_dxp, s_kq, s_sc);
    else
      derive_item_pair<ST, DD, false>(a, un, t, sm, v, s_plane, s_dxp, s_kq, s_sc);
  }
}

// Staged algebra kernel geometry: 32-point tasks (one warp each); a warp's buffer
// holds its task's staged slots and 24 KO sums per point, laid out as the blocked
// scratch holds them (scr_index).  MIXED stages all 138 slots in FP32 (20,736 B),
// 4 warps per CTA, 2 CTAs per SM (the register limit of the 254-register algebra).
// FP64 stages the 72 first derivatives and the KO sums (24,576 B) and reads the 66
// second derivatives, which the Ricci stage and the outputs use, from global memory
// after an L2 prefetch of their contiguous run: one-warp CTAs, 8 per SM (the register
// limit; staging all 138 slots fitted only 5).  In the upwind mode (ADV) the scratch
// also holds the 72 advective derivatives: MIXED stages them too (2 warps per CTA, 3
// CTAs per SM), FP64 reads them from global memory like the second derivatives.
constexpr int kStageW = 32;
template <typename ST, bool ADV = false>
struct StageCfg {
  static constexpr int kSlots = ADV ? kNumDerivs + 3 * kNumVars : kNumDerivs;  // 210 / 138
  // slots copied to shared memory: all in MIXED; in FP64 the 72 first derivatives (the
  // rest, prefetched into L2, is read from global memory), so 8 warps fit per SM
  static constexpr int kStaged = sizeof(ST) == 4 ? kSlots : 72;
  static constexpr int kWarps = sizeof(ST) == 4 ? (ADV ? 2 : 4) : 1;
  static constexpr int kThreads = 32 * kWarps;
  static constexpr int kMinBlocks = sizeof(ST) == 4 ? (ADV ? 3 : 2) : 8;
  static constexpr size_t kBytesPerWarp = (size_t)(kStaged + kNumVars) * kStageW * sizeof(ST);
  static constexpr size_t kSmemBytes = kWarps * kBytesPerWarp;
};

struct AlgebraArgs {
  const double* u[kNumVars];
  double* rhs[kNumVars];
  RkStage rk;
  const BlockDev* blocks;
  const UnitDev* units;
  const RangeDev* ranges;
  const void* dscr;
  const void* koscr;
  int32_t cap;
  int32_t range_base;
  AlgebraParams<double> prm64;
  AlgebraParams<float> prm32;
  double eta_const, eta_r0, eta_damping_exp, ko_sigma;
};

// Sommerfeld falloff / asymptotic value per VAR index (bssn/src/rhs.cpp:263-318).
__device__ __forceinline__ double bc_falloff(int v) {
  return (v >= 3 && v <= 5) || v >= 18 ? 2.0 : 1.0;
}
__device__ __forceinline__ double bc_asymptotic(int v) {
  return (v == 0 || v == 1 || v == 12 || v == 15 || v == 17) ? 1.0 : 0.0;
}

// Where an algebra thread reads its point's derivative slots and KO sums: straight
// from the scratch arrays in global memory, or from a copy its warp staged in
// shared memory (one 32-point column per slot).
template <typename ST>
struct GlobalScratch {
  const ST* d;       // slot 0 of the point: dscr + scr_index<kNumDerivs>(0, lp)
  const ST* ko;      // koscr + scr_index<kNumVars>(0, lp)
  __device__ __forceinline__ ST dv(int s) const { return __ldg(d + s * 32); }
  __device__ __forceinline__ double kov(int v) const { return (double)__ldg(ko + v * 32); }
};

template <typename ST, int STAGED>
struct SharedScratch {
  const ST* d;       // this lane's column: d[s * kStageW], slots s < STAGED
  const ST* ko;      // ko[v * kStageW]
  const ST* g;       // this lane's slot 0 in the scratch block (slots s >= STAGED)
  __device__ __forceinline__ ST dv(int s) const { return s < STAGED ? d[s * kStageW] : __ldg(g + s * kStageW); }
  __device__ __forceinline__ double kov(int v) const { return (double)ko[v * kStageW]; }
};

template <typename RT, class Src>
struct PointIn {
  const AlgebraArgs* a;
  int64_t pp;   // element index of the point in the variable arrays
  Src src;
  __device__ __forceinline__ RT u(int v) const { return (RT)__ldg(a->u[v] + pp); }
  __device__ __forceinline__ RT d(int s) const { return (RT)src.dv(s); }
};

// Stores the right-hand side k of variable v at element pp: to the RHS arrays
// (MODE RK_NONE) or through one RK4 stage update.  The mode is a template
// parameter so each instantiation is straight-line code: a run-time branch per
// output splits the generated algebra into basic blocks the scheduler cannot
// interleave across (measured: the algebra kernel ran 2x slower).
template <int MODE>
__device__ __forceinline__ void store_rhs(const AlgebraArgs& a, int v, int64_t pp, double k) {
  const RkStage& rk = a.rk;
  if constexpr (MODE == RK_LAST) {
    rk.base[v][pp] = rk.base[v][pp] + rk.acc[v][pp] + rk.w * k;
  } else if constexpr (MODE == RK_FIRST) {
    rk.acc[v][pp] = rk.w * k;
    rk.next[v][pp] = __ldg(rk.base[v] + pp) + rk.c * k;
  } else if constexpr (MODE == RK_MIDDLE) {
    rk.acc[v][pp] = rk.acc[v][pp] + rk.w * k;
    rk.next[v][pp] = __ldg(rk.base[v] + pp) + rk.c * k;
  } else {
    a.rhs[v][pp] = k;
  }
}

template <int MODE, class Src>
struct PointSink {
  const AlgebraArgs* a;
  int64_t pp;
  Src src;
  template <typename RT>
  __device__ __forceinline__ void put(int v, RT val) {
    // rhs += sigma * (ko_x + ko_y + ko_z), rounded as rhs.cpp:332-369 rounds it
    store_rhs<MODE>(*a, v, pp, __dadd_rn((double)val, __dmul_rn(a->ko_sigma, src.kov(v))));
  }
};

__device__ __forceinline__ void prefetch_l2_bulk(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// FP64 algebra as the two-part split of bssn_rhs_algebra_split.cuh
constexpr bool kSplitAlgebra64 = true;

// The right-hand side of interior point (i, j, k) (padded coordinates) of block B,
// inputs through `src`.
template <typename RT, int MODE, class Src, bool ADV = false>
__device__ __forceinline__ void algebra_point_at(const AlgebraArgs& a, const BlockDev& B, int i, int j,
                                                 int k, const Src& src) {
  const int nx = B.sz[0], ny = B.sz[1];
  const int64_t pp = B.offset + i + (int64_t)nx * (j + (int64_t)ny * k);
  // coordinates as bssnrhs forms them (pmin + i*h, two roundings, rhs.cpp:207-213)
  const double x = __dadd_rn(B.pmin[0], __dmul_rn((double)i, B.h[0]));
  const double y = __dadd_rn(B.pmin[1], __dmul_rn((double)j, B.h[1]));
  const double z = __dadd_rn(B.pmin[2], __dmul_rn((double)k, B.h[2]));
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
  const uint32_t bf = B.bflag;
  const bool on_face = ((bf & 1u) && i == 3) || ((bf & 2u) && i == nx - 4) ||
                       ((bf & 4u) && j == 3) || ((bf & 8u) && j == ny - 4) ||
                       ((bf & 16u) && k == 3) || ((bf & 32u) && k == B.sz[2] - 4);
  if (on_face) {
    // bssn_bcs (rhs.cpp:833-977) replaces the algebra on face planes; KO is added
    // afterwards (rhs.cpp:323-369).
    const double inv_r = 1.0 / sqrt(r2);
#pragma unroll 1
    for (int v = 0; v < kNumVars; ++v) {
      const double f = __ldg(a.u[v] + pp);
      const double dxf = (double)src.dv(3 * v + 0);
      const double dyf = (double)src.dv(3 * v + 1);
      const double dzf = (double)src.dv(3 * v + 2);
      double t = __dmul_rn(x, dxf);
      t = __dadd_rn(t, __dmul_rn(y, dyf));
      t = __dadd_rn(t, __dmul_rn(z, dzf));
      t = __dadd_rn(t, __dmul_rn(bc_falloff(v), __dsub_rn(f, bc_asymptotic(v))));
      const double val = __dmul_rn(-inv_r, t);
      store_rhs<MODE>(a, v, pp, __dadd_rn(val, __dmul_rn(a.ko_sigma, src.kov(v))));
    }
    return;
  }
  // eta damping, rhs.cpp:213-219
  const double r_coord = sqrt(r2);
  double eta = a.eta_const;
  if (r_coord >= a.eta_r0) eta *= pow(a.eta_r0 / r_coord, a.eta_damping_exp);

  PointIn<RT, Src> in{&a, pp, src};
  PointSink<MODE, Src> sink{&a, pp, src};
  const AlgebraParams<RT>* prm;
  if constexpr (sizeof(RT) == 8)
    prm = &a.prm64;
  else
    prm = &a.prm32;
  if constexpr (ADV) {
    bssn_rhs_algebra_adv<RT>(in, sink, *prm, (RT)eta);
  } else if constexpr (sizeof(RT) == 8 && kSplitAlgebra64) {
    // FP64: the algebra in two parts (the six At_rhs with the Ricci tensor, then the
    // rest), each with its own live set
    RhsAlgebraPart<0>::run<RT>(in, sink, *prm, (RT)eta);
    RhsAlgebraPart<1>::run<RT>(in, sink, *prm, (RT)eta);
  } else {
    bssn_rhs_algebra<RT>(in, sink, *prm, (RT)eta);
  }
}

// The same for interior point lpu (compact numbering) of unit `un`.
template <typename RT, int MODE, class Src, bool ADV = false>
__device__ __forceinline__ void algebra_point(const AlgebraArgs& a, const UnitDev& un, int lpu,
                                              const Src& src) {
  const BlockDev& B = a.blocks[un.block];
  const int I0 = B.sz[0] - 6, I1 = B.sz[1] - 6;
  const int lx = lpu % I0, rr = lpu / I0, ly = rr % I1, lz = rr / I1;
  algebra_point_at<RT, MODE, Src, ADV>(a, B, lx + 3, ly + 3, lz + 3 + un.k0, src);
}

// One CTA per range of up to 128 consecutive points of a unit, one thread per point,
// inputs loaded from global memory as the generated code needs them.
template <typename RT, typename ST, int MODE = RK_NONE>
__global__ void __launch_bounds__(kAlgebraThreads, 2)
bssn_algebra_kernel(const __grid_constant__ AlgebraArgs a) {
  const RangeDev rg = a.ranges[a.range_base + blockIdx.x];
  const UnitDev un = a.units[rg.unit];
  if (rg.count > 0) {
    // pull this CTA's scratch into L2 first, so the per-point loads below hit L2
    // instead of waiting on DRAM: the 32-point blocks its points fall in are one
    // contiguous run per array (every block starts on a 16-byte boundary)
    const int lp0 = (int)un.sbase + rg.start;
    const int b0 = lp0 >> 5, nblk = ((lp0 + rg.count - 1) >> 5) - b0 + 1;
    const char* pd = reinterpret_cast<const char*>(static_cast<const ST*>(a.dscr) + (size_t)b0 * kNumDerivs * 32);
    const char* pk = reinterpret_cast<const char*>(static_cast<const ST*>(a.koscr) + (size_t)b0 * kNumVars * 32);
    // in pieces of at most 4 KB (both runs are multiples of 16 bytes long)
    const uint32_t td = (uint32_t)nblk * kNumDerivs * 32 * sizeof(ST), tk = (uint32_t)nblk * kNumVars * 32 * sizeof(ST);
    const int nd = (int)((td + 4095) / 4096), nk = (int)((tk + 4095) / 4096);
    for (int k = threadIdx.x; k < nd + nk; k += kAlgebraThreads) {
      const bool dk = k < nd;
      const uint32_t off = 4096u * (uint32_t)(dk ? k : k - nd), tot = dk ? td : tk;
      prefetch_l2_bulk((dk ? pd : pk) + off, min(4096u, tot - off));
    }
  }
  if ((int)threadIdx.x >= rg.count) return;
  const int lpu = rg.start + threadIdx.x;
  const int lp = (int)un.sbase + lpu;
  const GlobalScratch<ST> src{static_cast<const ST*>(a.dscr) + scr_index<kNumDerivs>(0, lp),
                              static_cast<const ST*>(a.koscr) + scr_index<kNumVars>(0, lp)};
  algebra_point<RT, MODE>(a, un, lpu, src);
}


__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Staged algebra kernel: persistent warps, each taking 32-point tasks
// (quarters of a range) round-robin.  A task first copies its points' 138 slots
// and 24 KO sums -- one contiguous block each in the blocked scratch -- into the
// warp's shared-memory buffer with lane-strided 16-byte cp.async (the planner
// starts every unit's scratch run on a 32-point boundary and pads the scratch, so
// the copies are aligned and in bounds) and prefetches the 24 state values into L2,
// then runs the algebra reading shared memory: the loads that kept the
// one-CTA-per-range version waiting on L2/DRAM become shared-memory loads, and while
// one warp waits for its copies the others compute.
template <typename ST, int MODE, bool ADV = false>
__global__ void __launch_bounds__(StageCfg<ST, ADV>::kThreads, StageCfg<ST, ADV>::kMinBlocks)
bssn_algebra_staged_kernel(const __grid_constant__ AlgebraArgs a, int ntasks) {
  using Cfg = StageCfg<ST, ADV>;
  using RT = ST;  // FP32 algebra in MIXED, FP64 in FP64
  extern __shared__ __align__(16) unsigned char s_stage[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  ST* sd = reinterpret_cast<ST*>(s_stage + warp * Cfg::kBytesPerWarp);
  ST* sk = reinterpret_cast<ST*>(s_stage + warp * Cfg::kBytesPerWarp +
                                 Cfg::kStaged * kStageW * sizeof(ST));
  const int nwarps = gridDim.x * Cfg::kWarps;
  for (int t = blockIdx.x * Cfg::kWarps + warp; t < ntasks; t += nwarps) {
    const RangeDev rg = a.ranges[a.range_base + (t >> 2)];
    const int start = (t & 3) * kStageW;
    if (start >= rg.count) continue;
    const UnitDev un = a.units[rg.unit];
    const int lp0 = (int)un.sbase + rg.start + start;  // multiple of 32
    const int lpu = rg.start + start + lane;
    const bool valid = start + lane < rg.count;
    if (valid) {
      const BlockDev& B = a.blocks[un.block];
      const int I0 = B.sz[0] - 6, I1 = B.sz[1] - 6;
      const int lx = lpu % I0, rr = lpu / I0, ly = rr % I1, lz = rr / I1;
      const int64_t pp = B.offset + (lx + 3) + (int64_t)B.sz[0] * ((ly + 3) + (int64_t)B.sz[1] * (lz + 3 + un.k0));
#pragma unroll
      for (int v = 0; v < kNumVars; ++v) prefetch_l2(a.u[v] + pp);
      if constexpr (MODE == RK_MIDDLE || MODE == RK_LAST) {
        // the stage update reads u^n and the accumulator at every output
#pragma unroll
        for (int v = 0; v < kNumVars; ++v) {
          prefetch_l2(a.rk.base[v] + pp);
          prefetch_l2(a.rk.acc[v] + pp);
        }
      }
    }
    __syncwarp();  // every lane is done reading the previous task's buffer
    {
      // the task's slots and KO sums are one contiguous block each in the scratch
      // (scr_index; lp0 is a multiple of 32), laid out exactly as the buffer wants
      // them: copy both in 16-byte pieces, lane-strided
      constexpr int ND = Cfg::kStaged * kStageW * (int)sizeof(ST) / 16, NK = kNumVars * kStageW * (int)sizeof(ST) / 16;
      const char* d = reinterpret_cast<const char*>(static_cast<const ST*>(a.dscr) + (size_t)lp0 * Cfg::kSlots);
      const char* ko = reinterpret_cast<const char*>(static_cast<const ST*>(a.koscr) + (size_t)lp0 * kNumVars);
#pragma unroll 6
      for (int k = lane; k < ND; k += 32) cp_async16(reinterpret_cast<char*>(sd) + 16 * k, d + 16 * k);
#pragma unroll 4
      for (int k = lane; k < NK; k += 32) cp_async16(reinterpret_cast<char*>(sk) + 16 * k, ko + 16 * k);
      if constexpr (Cfg::kStaged < Cfg::kSlots) {
        // the unstaged slots: one contiguous run after the staged ones, into L2
        constexpr uint32_t kRest = (Cfg::kSlots - Cfg::kStaged) * kStageW * sizeof(ST);
        constexpr int kPieces = (int)((kRest + 4095) / 4096);
        static_assert(kPieces <= 32, "one piece per lane");
        if (lane < kPieces) {
          const uint32_t off = 4096u * (uint32_t)lane;
          prefetch_l2_bulk(d + (size_t)ND * 16 + off, min(4096u, kRest - off));
        }
      }
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncwarp();  // the copies of every lane are visible to the whole warp
    if (valid) {
      using Src = SharedScratch<ST, Cfg::kStaged>;
      const Src src{sd + lane, sk + lane,
                    static_cast<const ST*>(a.dscr) + (size_t)lp0 * Cfg::kSlots + lane};
      algebra_point<RT, MODE, Src, ADV>(a, un, lpu, src);
    }
  }
}

}  // namespace b200bssn
