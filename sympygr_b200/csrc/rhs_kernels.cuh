// The two kernels of one right-hand-side evaluation of a chunk of blocks.
//
//  bssn_derivs_kernel   one CTA per (x-y tile of a unit, variable): stages the
//                       variable's tile with a 4-point halo in shared memory and
//                       writes, per interior point, the variable's first
//                       derivatives, its second derivatives when it has them
//                       (mixed ones as compositions D_y(D_x u), D_z(D_x u),
//                       D_z(D_y u), exactly as bssn/scripts/bssnrhs_derivs.h
//                       composes them), and the sum of its three KO terms, into the
//                       chunk's derivative scratch.
//  bssn_algebra_kernel  one thread per interior point: the generated BSSN algebra
//                       (or, on a flagged face plane, the Sommerfeld value of
//                       bssn/src/rhs.cpp:833-977), plus sigma times the KO sum
//                       (bssn/src/rhs.cpp:332-369), written to the RHS arrays.
#pragma once
#include <stdint.h>

#include "generated/bssn_rhs_algebra.cuh"
#include "plan_types.h"
#include "stencils.cuh"

namespace b200bssn {

constexpr int kSX = kTileX + 2 * kHalo, kSY = kTileY + 2 * kHalo, kSZ = kTileZ + 2 * kHalo;
constexpr int kDerivSmemDoubles = kSZ * kSY * kSX + kSZ * kSY * kTileX + kSZ * kTileY * kTileX;
constexpr size_t kDerivSmemBytes = sizeof(double) * kDerivSmemDoubles;

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
  void* dscr;        // kNumDerivs slots of `cap` values (double or float)
  double* koscr;     // kNumVars slots of `cap` doubles
  int64_t cap;
  int32_t tile_base;
};

template <typename ST>
__global__ void __launch_bounds__(kDerivThreads)
bssn_derivs_kernel(const __grid_constant__ DerivArgs a) {
  extern __shared__ double smem[];
  double* s_u = smem;                        // [kSZ][kSY][kSX]
  double* s_dx = s_u + kSZ * kSY * kSX;      // [kSZ][kSY][kTileX]
  double* s_dy = s_dx + kSZ * kSY * kTileX;  // [kSZ][kTileY][kTileX]

  const TileDev t = a.tiles[a.tile_base + blockIdx.x];
  const UnitDev un = a.units[t.unit];
  const BlockDev B = a.blocks[un.block];
  const int v = blockIdx.y;
  const int q = dd_index(v);
  const int nx = B.sz[0], ny = B.sz[1], nz = B.sz[2];
  const int I0 = nx - 6, I1 = ny - 6;
  const int i0 = 3 + t.i0, j0 = 3 + t.j0, k0 = 3 + un.k0;
  const int ex = t.ex, ey = t.ey, ez = un.nz;
  const int ox = i0 - kHalo, oy = j0 - kHalo, oz = k0 - kHalo;  // smem origin (padded coords)
  const int xlo = max(0, ox), xhi = min(nx, i0 + ex + kHalo);
  const int ylo = max(0, oy), yhi = min(ny, j0 + ey + kHalo);
  const int zlo = max(0, oz), zhi = min(nz, k0 + ez + kHalo);
  const int lx = xhi - xlo, ly = yhi - ylo, lz = zhi - zlo;

  const double* __restrict__ f = a.u[v] + B.offset;
  for (int idx = threadIdx.x; idx < lx * ly * lz; idx += blockDim.x) {
    const int x = idx % lx, r = idx / lx, y = r % ly, z = r / ly;
    const int gi = xlo + x, gj = ylo + y, gk = zlo + z;
    s_u[((gk - oz) * kSY + (gj - oy)) * kSX + (gi - ox)] =
        __ldg(f + gi + (int64_t)nx * (gj + (int64_t)ny * gk));
  }
  __syncthreads();

  const LineScales cx = make_line_scales(B.h[0]);
  const LineScales cy = make_line_scales(B.h[1]);
  const LineScales cz = make_line_scales(B.h[2]);
  const uint32_t bf = B.bflag;
  const bool lox = bf & 1u, hix = bf & 2u, loy = bf & 4u, hiy = bf & 8u, loz = bf & 16u,
             hiz = bf & 32u;

  if (q >= 0) {
    // D_x on the tile's x range over the y/z halo (deriv64_x covers all j,k,
    // bssn/src/derivs.cpp:2067-2068), then D_y on the tile's x-y range over the z
    // halo (deriv64_y covers all k, :2199-2202).
    for (int idx = threadIdx.x; idx < ex * ly * lz; idx += blockDim.x) {
      const int x = idx % ex, r = idx / ex, y = r % ly, z = r / ly;
      const int gi = i0 + x, gj = ylo + y, gk = zlo + z;
      const double* pu = &s_u[((gk - oz) * kSY + (gj - oy)) * kSX + (gi - ox)];
      s_dx[((gk - oz) * kSY + (gj - oy)) * kTileX + x] = line_d1(pu, 1, gi, nx, lox, hix, cx);
    }
    for (int idx = threadIdx.x; idx < ex * ey * lz; idx += blockDim.x) {
      const int x = idx % ex, r = idx / ex, y = r % ey, z = r / ey;
      const int gi = i0 + x, gj = j0 + y, gk = zlo + z;
      const double* pu = &s_u[((gk - oz) * kSY + (gj - oy)) * kSX + (gi - ox)];
      s_dy[((gk - oz) * kTileY + y) * kTileX + x] = line_d1(pu, kSX, gj, ny, loy, hiy, cy);
    }
    __syncthreads();
  }

  ST* __restrict__ dscr = static_cast<ST*>(a.dscr);
  const int64_t cap = a.cap;
  for (int idx = threadIdx.x; idx < ex * ey * ez; idx += blockDim.x) {
    const int x = idx % ex, r = idx / ex, y = r % ey, z = r / ey;
    const int gi = i0 + x, gj = j0 + y, gk = k0 + z;
    const double* pu = &s_u[((gk - oz) * kSY + (gj - oy)) * kSX + (gi - ox)];
    const int64_t lp = un.sbase + (gi - 3) + (int64_t)I0 * ((gj - 3) + (int64_t)I1 * (gk - k0));

    double d0, d1;
    const double* pdx = &s_dx[((gk - oz) * kSY + (gj - oy)) * kTileX + x];
    const double* pdy = &s_dy[((gk - oz) * kTileY + y) * kTileX + x];
    if (q >= 0) {
      d0 = *pdx;
      d1 = *pdy;
    } else {
      d0 = line_d1(pu, 1, gi, nx, lox, hix, cx);
      d1 = line_d1(pu, kSX, gj, ny, loy, hiy, cy);
    }
    const double d2 = line_d1(pu, kSX * kSY, gk, nz, loz, hiz, cz);
    // rhs.cpp:332-369 adds grad_0 + grad_1 + grad_2 of the KO pass in this order
    const double ko = __dadd_rn(__dadd_rn(line_ko(pu, 1, gi, nx, lox, hix, cx),
                                          line_ko(pu, kSX, gj, ny, loy, hiy, cy)),
                                line_ko(pu, kSX * kSY, gk, nz, loz, hiz, cz));
    dscr[(3 * v + 0) * cap + lp] = (ST)d0;
    dscr[(3 * v + 1) * cap + lp] = (ST)d1;
    dscr[(3 * v + 2) * cap + lp] = (ST)d2;
    a.koscr[v * cap + lp] = ko;
    if (q >= 0) {
      const int s0 = 72 + 6 * q;
      dscr[(s0 + 0) * cap + lp] = (ST)line_d2(pu, 1, gi, nx, lox, hix, cx);
      dscr[(s0 + 1) * cap + lp] = (ST)line_d1(pdx, kTileX, gj, ny, loy, hiy, cy);
      dscr[(s0 + 2) * cap + lp] = (ST)line_d1(pdx, kSY * kTileX, gk, nz, loz, hiz, cz);
      dscr[(s0 + 3) * cap + lp] = (ST)line_d2(pu, kSX, gj, ny, loy, hiy, cy);
      dscr[(s0 + 4) * cap + lp] = (ST)line_d1(pdy, kTileY * kTileX, gk, nz, loz, hiz, cz);
      dscr[(s0 + 5) * cap + lp] = (ST)line_d2(pu, kSX * kSY, gk, nz, loz, hiz, cz);
    }
  }
}

struct AlgebraArgs {
  const double* u[kNumVars];
  double* rhs[kNumVars];
  const BlockDev* blocks;
  const UnitDev* units;
  const RangeDev* ranges;
  const void* dscr;
  const double* koscr;
  int64_t cap;
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

template <typename RT, typename ST>
struct PointIn {
  const AlgebraArgs* a;
  int64_t pp;   // element index of the point in the variable arrays
  int64_t lp;   // scratch index
  __device__ __forceinline__ RT u(int v) const { return (RT)__ldg(a->u[v] + pp); }
  __device__ __forceinline__ RT d(int s) const {
    return (RT)__ldg(static_cast<const ST*>(a->dscr) + s * a->cap + lp);
  }
};

struct PointSink {
  const AlgebraArgs* a;
  int64_t pp, lp;
  template <typename RT>
  __device__ __forceinline__ void put(int v, RT val) {
    // rhs += sigma * (ko_x + ko_y + ko_z), rounded as rhs.cpp:332-369 rounds it
    a->rhs[v][pp] = __dadd_rn((double)val, __dmul_rn(a->ko_sigma, __ldg(a->koscr + v * a->cap + lp)));
  }
};

template <typename RT, typename ST>
__global__ void __launch_bounds__(kAlgebraThreads, 2)
bssn_algebra_kernel(const __grid_constant__ AlgebraArgs a) {
  const RangeDev rg = a.ranges[a.range_base + blockIdx.x];
  if ((int)threadIdx.x >= rg.count) return;
  const UnitDev un = a.units[rg.unit];
  const BlockDev& B = a.blocks[un.block];
  const int nx = B.sz[0], ny = B.sz[1];
  const int I0 = nx - 6, I1 = ny - 6;
  const int lpu = rg.start + threadIdx.x;
  const int lx = lpu % I0, rr = lpu / I0, ly = rr % I1, lz = rr / I1;
  const int i = lx + 3, j = ly + 3, k = lz + 3 + un.k0;
  const int64_t pp = B.offset + i + (int64_t)nx * (j + (int64_t)ny * k);
  const int64_t lp = un.sbase + lpu;
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
    const ST* ds = static_cast<const ST*>(a.dscr);
#pragma unroll 1
    for (int v = 0; v < kNumVars; ++v) {
      const double f = __ldg(a.u[v] + pp);
      const double dxf = (double)__ldg(ds + (3 * v + 0) * a.cap + lp);
      const double dyf = (double)__ldg(ds + (3 * v + 1) * a.cap + lp);
      const double dzf = (double)__ldg(ds + (3 * v + 2) * a.cap + lp);
      double t = __dmul_rn(x, dxf);
      t = __dadd_rn(t, __dmul_rn(y, dyf));
      t = __dadd_rn(t, __dmul_rn(z, dzf));
      t = __dadd_rn(t, __dmul_rn(bc_falloff(v), __dsub_rn(f, bc_asymptotic(v))));
      const double val = __dmul_rn(-inv_r, t);
      a.rhs[v][pp] = __dadd_rn(val, __dmul_rn(a.ko_sigma, __ldg(a.koscr + v * a.cap + lp)));
    }
    return;
  }
  // eta damping, rhs.cpp:213-219
  const double r_coord = sqrt(r2);
  double eta = a.eta_const;
  if (r_coord >= a.eta_r0) eta *= pow(a.eta_r0 / r_coord, a.eta_damping_exp);

  PointIn<RT, ST> in{&a, pp, lp};
  PointSink sink{&a, pp, lp};
  if constexpr (sizeof(RT) == 8) {
    bssn_rhs_algebra<RT>(in, sink, a.prm64, (RT)eta);
  } else {
    bssn_rhs_algebra<RT>(in, sink, a.prm32, (RT)eta);
  }
}

}  // namespace b200bssn
