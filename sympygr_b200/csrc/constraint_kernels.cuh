// Hamiltonian and momentum constraints on the derivative scratch.
//
// The reference evaluates the constraints on the CPU in `physical_constraints`
// (bssn/CodeGen/physcon.cpp:12-1398, generated from GR/constraints.py:166-177): it
// materialises first derivatives of chi, Gt, K, gt, At and second derivatives of gt
// and chi with the same 6th-order operators as bssnrhs, then evaluates
//   ham   = chi igt^jk R_jk - A_ij A^ij + 2/3 K^2
//   mom_i = ...                                   (GR/constraints.py:170-177)
// at every interior point. Here the derivatives come from the derivative kernel
// (the derivative stage, whose 138 slots include all 93 the constraints read), and
// one thread per interior point runs the generated constraint algebra
// (generated/bssn_constraints_algebra.cuh).
//
// Outputs, each optional: the four constraint fields at the interior points of the
// caller's arrays (indexed like the state), and per block the sums of squares and
// the maxima of |ham|, |mom0..2| over its interior points (8 doubles per block,
// accumulated with one atomic per CTA and constraint; a non-finite value makes the
// maximum NaN, so the norms double as a finiteness check).
#pragma once

#include "plan_types.h"
#include "generated/bssn_constraints_algebra.cuh"

namespace b200bssn {

constexpr int kNumConstraints = 4;  // ham, mom0, mom1, mom2

struct ConstraintArgs {
  const double* u[kNumVars];
  double* con[kNumConstraints];  // all null: fields not written
  double* norms;                 // [nblocks][8] or null
  const BlockDev* blocks;
  const UnitDev* units;
  const RangeDev* ranges;
  const void* dscr;  // derivative slots, layout scr_index with nslots slots per point
  int32_t cap;
  int32_t nslots;
  int32_t range_base;
};

template <typename RT, typename ST>
struct ConstraintIn {
  const ConstraintArgs* a;
  int64_t pp;
  int lp;
  __device__ __forceinline__ RT u(int v) const { return (RT)__ldg(a->u[v] + pp); }
  __device__ __forceinline__ RT d(int s) const {
    return (RT)__ldg(static_cast<const ST*>(a->dscr) + scr_index(a->nslots, s, lp));
  }
};

template <typename RT>
struct ConstraintSink {
  RT val[kNumConstraints];
  __device__ __forceinline__ void put(int c, RT v) { val[c] = v; }
};

// non-negative doubles (and NaN with the sign bit clear) order like their bit patterns
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr),
            (unsigned long long)__double_as_longlong(v));
}

template <typename RT, typename ST>
__global__ void __launch_bounds__(kAlgebraThreads)
bssn_constraints_kernel(const __grid_constant__ ConstraintArgs a) {
  const RangeDev rg = a.ranges[a.range_base + blockIdx.x];
  const UnitDev un = a.units[rg.unit];
  const BlockDev& B = a.blocks[un.block];
  const bool active = (int)threadIdx.x < rg.count;
  if (sizeof(ST) == 8 && rg.count > 0) {
    // FP64 (latency bound at 255 registers): pull the run's scratch into L2 first, so
    // the per-point loads below hit L2; its 32-point blocks are one contiguous run
    // (16-byte aligned), prefetched in pieces of at most 4 KB.  (MIXED, closer to the
    // DRAM bound, lost 3 % to the extra instructions.)
    const int lp0 = (int)un.sbase + rg.start;
    const int b0 = lp0 >> 5, nblk = ((lp0 + rg.count - 1) >> 5) - b0 + 1;
    const char* pd = reinterpret_cast<const char*>(static_cast<const ST*>(a.dscr) + (size_t)b0 * a.nslots * 32);
    const uint32_t td = (uint32_t)nblk * (uint32_t)a.nslots * 32u * (uint32_t)sizeof(ST);
    const int npc = (int)((td + 4095u) / 4096u);
    for (int k = threadIdx.x; k < npc; k += kAlgebraThreads)
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(pd + 4096u * (uint32_t)k),
                   "r"(min(4096u, td - 4096u * (uint32_t)k))
                   : "memory");
  }
  double sq[kNumConstraints] = {0.0, 0.0, 0.0, 0.0};
  double mx[kNumConstraints] = {0.0, 0.0, 0.0, 0.0};
  if (active) {
    const int nx = B.sz[0], ny = B.sz[1];
    const int I0 = nx - 6, I1 = ny - 6;
    const int lpu = rg.start + threadIdx.x;
    const int lx = lpu % I0, rr = lpu / I0, ly = rr % I1, lz = rr / I1;
    const int64_t pp =
        B.offset + (lx + 3) + (int64_t)nx * ((ly + 3) + (int64_t)ny * (lz + 3 + un.k0));
    if (sizeof(ST) == 8) {
#pragma unroll
      for (int v = 0; v < kNumVars; ++v) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.u[v] + pp));
    }
    ConstraintIn<RT, ST> in{&a, pp, (int)un.sbase + lpu};
    ConstraintSink<RT> sink;
    bssn_constraints_algebra<RT>(in, sink);
#pragma unroll
    for (int c = 0; c < kNumConstraints; ++c) {
      const double v = (double)sink.val[c];
      if (a.con[c]) a.con[c][pp] = v;
      sq[c] = v * v;
      mx[c] = fabs(v);
    }
  }
  if (!a.norms) return;
  // CTA reduction: warp shuffles, then one value per warp through shared memory
  __shared__ double s_red[kAlgebraThreads / 32][2 * kNumConstraints];
#pragma unroll
  for (int c = 0; c < kNumConstraints; ++c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sq[c] += __shfl_xor_sync(0xffffffffu, sq[c], o);
      const double m = __shfl_xor_sync(0xffffffffu, mx[c], o);
      mx[c] = (m > mx[c] || m != m) ? m : mx[c];
    }
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int c = 0; c < kNumConstraints; ++c) {
      s_red[w][c] = sq[c];
      s_red[w][kNumConstraints + c] = mx[c];
    }
  }
  __syncthreads();
  if (threadIdx.x < 2 * kNumConstraints) {
    const int c = threadIdx.x;
    double r = s_red[0][c];
    for (int k = 1; k < kAlgebraThreads / 32; ++k) {
      const double t = s_red[k][c];
      r = c < kNumConstraints ? r + t : ((t > r || t != t) ? t : r);
    }
    double* dst = a.norms + (size_t)un.block * (2 * kNumConstraints) + c;
    if (c < kNumConstraints)
      atomicAdd(dst, r);
    else
      atomic_max_nonneg(dst, fabs(r));
  }
}

}  // namespace b200bssn
