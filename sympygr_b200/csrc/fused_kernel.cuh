// Single-pass right-hand side: one persistent kernel for a whole evaluation, with
// the derivative scratch kept in a ring of tile-slab slots small enough to stay in
// the 126 MB L2 instead of a full scratch array in HBM.
//
// Work units (plan order, see b200bssn.cu):
//   tile-slab T  a 16x8 column tile of a block over a z-slab of at most kFusedSlab
//                interior planes; it owns ring slot T % nring while in flight
//   item (T, v)  the derivative stage of variable v on tile-slab T (derive_item, the
//                same streaming stencil as the two-pass kernels), written into the
//                slot in the blocked layout of 32-point runs: point (tx, ty, z) of the
//                tile is lp = slot * kFusedSlotPts + tx + 16 ty + 128 z
//   group (T, z) the algebra of plane z of tile-slab T: warp w takes rows 2w, 2w+1
//                (one 32-point run), copies its 138 slots into shared memory and runs
//                the generated algebra, the Sommerfeld faces and the KO term
//                (algebra_point_at), storing the RHS or an RK4 stage update
//
// Scheduling (thread 0 of each CTA): a CTA claims, with a compare-and-swap on the
// global counter, exactly the next algebra group if its tile-slab has all 24
// items done, else exactly the next item if its tile-slab's ring slot is free
// (the previous tile-slab in that slot has all its groups done).  A CTA therefore
// only ever holds work it can run at once; items and groups are claimed in order,
// so the earliest unfinished tile-slab can always progress and no set of CTAs can
// wait on each other.  When nothing can be claimed the CTA sleeps briefly and
// retries; every such wait is bounded by the global timer (kFusedWaitNs), after
// which the kernel records an error word and every CTA returns.
//
// Memory ordering: a producer's threads fence and meet at a CTA barrier, then
// thread 0 increments the tile-slab's done counter; a consumer reads the counter,
// fences, and reads the slot through L2 only (cp.async.cg and ld.global.cg: the
// slot was written by other SMs, and L1 is not coherent).  After a run's slots and
// KO sums are consumed its 128-byte lines are dropped from L2 without a write-back
// (discard.global.L2), so the ring's traffic stays on chip.
#pragma once
#include "rhs_kernels.cuh"

namespace b200bssn {

constexpr int kFusedThreads = 128;                              // 4 warps: one derivative item or one group
constexpr int kFusedMinBlocks = 3;                              // CTAs per SM (168 registers)
constexpr unsigned long long kFusedWaitNs = 2000000000ull;      // 2 s per wait, then an error
constexpr size_t kFusedStageBytes = (size_t)kNumDerivs * kStageW * sizeof(float);  // per warp
constexpr size_t kFusedSmemBytes = 4 * kFusedStageBytes;        // 70,656 B (derivative buffers alias it)
static_assert(4 * kPlane * sizeof(double) + 2 * kDxRows * kTileX * sizeof(double) +
                      (kHalo + 1) * kDerivThreads * sizeof(double) <= kFusedSmemBytes,
              "the derivative item's buffers fit in the algebra staging area");
static_assert(kFusedThreads == kDerivThreads, "one CTA shape for both roles");

// Device words of one evaluation, zeroed before the launch:
//   [0] next item, [1] next group, [2] error (1: a wait timed out), [3] unused,
//   done[ntiles] (items finished per tile-slab), used[ntiles] (groups finished),
//   gen[nring] (slot s is free for tile-slab T when gen[s] == T / nring)
struct FusedArgs {
  DerivArgs d;        // state, blocks; dscr/koscr = the ring (MIXED: float)
  AlgebraArgs a;      // state, RHS or RK4 stage, parameters
  const FusedTileDev* tiles;
  const int32_t* group_tile;  // tile-slab of each group
  int32_t ntiles, ngroups, nring;
  int* sync;
};

__device__ __forceinline__ int ld_relaxed(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void discard_l2_line(const void* p) {
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

enum FusedRole : int { FR_EXIT = 0, FR_ITEM = 1, FR_GROUP = 2 };

// Thread 0: the next unit of work for this CTA (see the scheduling note above).
__device__ __forceinline__ void fused_schedule(const FusedArgs& f, int* role, int* idx) {
  int* const next_item = f.sync + 0;
  int* const next_group = f.sync + 1;
  int* const err = f.sync + 2;
  const int* const done = f.sync + 4;
  const int* const gen = f.sync + 4 + 2 * f.ntiles;
  const int nitems = f.ntiles * kNumVars;
  unsigned long long t0 = 0;
  unsigned sleep = 32;
  for (;;) {
    if (ld_relaxed(err)) break;
    const int g = ld_relaxed(next_group);
    if (g >= f.ngroups) break;  // every group claimed (so every item was claimed before)
    const int tg = __ldg(f.group_tile + g);
    if (ld_relaxed(done + tg) == kNumVars) {
      if (atomicCAS(next_group, g, g + 1) == g) {
        __threadfence();  // the tile-slab's slots are read after its done count
        *role = FR_GROUP;
        *idx = g;
        return;
      }
      sleep = 32;
      continue;  // lost the race: look again at once
    }
    const int d = ld_relaxed(next_item);
    if (d < nitems) {
      const int T = d / kNumVars;
      if (ld_relaxed(gen + T % f.nring) == T / f.nring) {
        if (atomicCAS(next_item, d, d + 1) == d) {
          __threadfence();  // the slot's previous readers are done before it is rewritten
          *role = FR_ITEM;
          *idx = d;
          return;
        }
        sleep = 32;
        continue;
      }
    }
    // nothing can be claimed now: the work that unblocks it is running on other CTAs
    const unsigned long long now = global_ns();
    if (t0 == 0) {
      t0 = now;
    } else if (now - t0 > kFusedWaitNs) {
      atomicExch(err, 1);
      break;
    }
    __nanosleep(sleep);
    sleep = min(sleep * 2, 1024u);
  }
  *role = FR_EXIT;
  *idx = 0;
}

// Slots from this warp's shared-memory copy, KO sums straight from the ring in L2.
struct FusedScratch {
  const float* d;   // this lane's column: d[s * kStageW]
  const float* ko;  // this lane's KO sums in the ring: ko[v * 32]
  __device__ __forceinline__ float dv(int s) const { return d[s * kStageW]; }
  __device__ __forceinline__ double kov(int v) const { return (double)__ldcg(ko + v * 32); }
};

template <int MODE>
__global__ void __launch_bounds__(kFusedThreads, kFusedMinBlocks)
bssn_fused_kernel(const __grid_constant__ FusedArgs f) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ LineScales s_sc[3];
  __shared__ int s_role, s_idx;
  double(*s_plane)[kPlane] = reinterpret_cast<double(*)[kPlane]>(smem);
  double* s_dxp = reinterpret_cast<double*>(smem + 4 * kPlane * sizeof(double));
  double* s_kq = s_dxp + 2 * kDxRows * kTileX;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* const done = f.sync + 4;
  int* const used = f.sync + 4 + f.ntiles;
  int* const gen = f.sync + 4 + 2 * f.ntiles;

  for (;;) {
    if (threadIdx.x == 0) fused_schedule(f, &s_role, &s_idx);
    __syncthreads();
    const int role = s_role, idx = s_idx;
    if (role == FR_EXIT) break;
    if (role == FR_ITEM) {
      const int T = idx / kNumVars, v = idx % kNumVars;
      const FusedTileDev ft = f.tiles[T];
      const UnitDev un{ft.block, ft.k0, ft.nz, 0, 0};
      const TileDev t{0, ft.i0, ft.j0, ft.ex, ft.ey};
      const ScratchMap sm{(T % f.nring) * kFusedSlotPts, kTileX, kTileX * kTileY};
      const bool cl = item_has_closure(f.d.blocks[ft.block], un, t);
      if (dd_index(v) >= 0) {
        if (cl)
          derive_item<float, true, false, true>(f.d, un, t, sm, v, s_plane, s_dxp, s_kq, s_sc);
        else
          derive_item<float, true, false, false>(f.d, un, t, sm, v, s_plane, s_dxp, s_kq, s_sc);
      } else {
        if (cl)
          derive_item<float, false, false, true>(f.d, un, t, sm, v, s_plane, s_dxp, s_kq, s_sc);
        else
          derive_item<float, false, false, false>(f.d, un, t, sm, v, s_plane, s_dxp, s_kq, s_sc);
      }
      __threadfence();  // this thread's slot writes, before the done count
      __syncthreads();
      if (threadIdx.x == 0) atomicAdd(done + T, 1);
    } else {
      const int g = idx;
      const int T = __ldg(f.group_tile + g);
      const FusedTileDev ft = f.tiles[T];
      const int z = g - ft.group_base;
      const int run = (T % f.nring) * (kFusedSlotPts / 32) + z * 4 + warp;  // 32-point run in the ring
      const int tx = lane & 15, ty = 2 * warp + (lane >> 4);
      const bool any = 2 * warp < ft.ey;
      const bool valid = tx < ft.ex && ty < ft.ey;
      float* sd = reinterpret_cast<float*>(smem + warp * kFusedStageBytes);
      const float* gd = static_cast<const float*>(f.d.dscr) + (size_t)run * kNumDerivs * 32;
      const float* gk = static_cast<const float*>(f.d.koscr) + (size_t)run * kNumVars * 32;
      const BlockDev& B = f.a.blocks[ft.block];
      const int i = 3 + ft.i0 + tx, j = 3 + ft.j0 + ty, k = 3 + ft.k0 + z;
      if (any) {
        if (valid) {
          const int64_t pp = B.offset + i + (int64_t)B.sz[0] * (j + (int64_t)B.sz[1] * k);
#pragma unroll
          for (int v = 0; v < kNumVars; ++v) prefetch_l2(f.a.u[v] + pp);
          if constexpr (MODE == RK_MIDDLE || MODE == RK_LAST) {
#pragma unroll
            for (int v = 0; v < kNumVars; ++v) {
              prefetch_l2(f.a.rk.base[v] + pp);
              prefetch_l2(f.a.rk.acc[v] + pp);
            }
          }
        }
        constexpr int ND = (int)(kFusedStageBytes / 16);
#pragma unroll 6
        for (int q = lane; q < ND; q += 32)
          cp_async16(reinterpret_cast<char*>(sd) + 16 * q, reinterpret_cast<const char*>(gd) + 16 * q);
        cp_async_commit();
        cp_async_wait<0>();
        __syncwarp();
        // the run's slots are in shared memory: drop their lines from L2 unwritten
        for (int q = lane; q < (int)(kFusedStageBytes / 128); q += 32)
          discard_l2_line(reinterpret_cast<const char*>(gd) + 128 * q);
        if (valid) {
          const FusedScratch src{sd + lane, gk + lane};
          algebra_point_at<float, MODE, FusedScratch, false>(f.a, B, i, j, k, src);
        }
        __syncwarp();  // every lane has read its KO sums
        if (lane < kNumVars) discard_l2_line(gk + lane * 32);
      }
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) {
        if (atomicAdd(used + T, 1) == ft.nz - 1) {
          __threadfence();
          atomicExch(gen + T % f.nring, T / f.nring + 1);  // the slot is free for T + nring
        }
      }
    }
    __syncthreads();  // s_role / s_idx and the shared buffers are free for the next unit
  }
}

}  // namespace b200bssn
