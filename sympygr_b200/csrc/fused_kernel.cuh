// Single-pass right-hand side: one persistent kernel for a whole evaluation, with
// the derivative scratch in a ring of tile-slab slots instead of a full scratch array
// in HBM: each slot is reused as soon as its tile-slab's algebra is done, so the lines
// written are read back (mostly from L2) while they are fresh.  The default ring has
// 128 slots (256 MB); 32 slots (64 MB) fit the 126 MB L2 but leave items waiting for
// free slots (measured slower).
//
// Work units (plan order, see b200bssn.cu):
//   tile-slab T  a 16x8 column tile of a block over a z-slab of at most kFusedSlab
//                interior planes; it owns ring slot T % nring while in flight
//   item (T, v)  the derivative stage of variable v on tile-slab T (derive_item, the
//                same streaming stencil as the two-pass kernels), written into the
//                slot in the blocked layout of 32-point runs: point (tx, ty, z) of the
//                tile is lp = slot * kFusedSlotPts + tx + 16 ty + 128 z
//   planes of T  the algebra of plane z of tile-slab T: warp w takes rows 2w, 2w+1
//                (one 32-point run), copies its 138 slots into shared memory and runs
//                the generated algebra, the Sommerfeld faces and the KO term
//                (algebra_point_at), storing the RHS or an RK4 stage update; a claim
//                covers kFusedPlanes planes
//
// Scheduling (warp 0 of each CTA, all 32 lanes together):
//   * algebra first: the lanes look at the next 32 tile-slabs from the algebra hint
//     (the first tile-slab whose algebra is not all claimed) at once; a tile-slab whose
//     24 items are done hands out its planes kFusedPlanes at a time through its own
//     fetch-and-add counter, so no single counter serialises the claims;
//   * else the next item, by fetch-and-add on the item counter; if its tile-slab's
//     ring slot is not free yet (the tile-slab nring earlier still has algebra
//     running) the CTA keeps the item and takes algebra work until the slot frees.
// Items are handed out in order, so the oldest unfinished tile-slab never waits on a
// slot (its predecessor in the slot is older still, hence finished), its items
// complete, and its algebra can be claimed by any CTA: work always progresses,
// whether or not every CTA of the grid is resident.  A CTA with nothing to claim
// sleeps briefly and retries; every wait is bounded by the global timer
// (kFusedWaitNs), after which the kernel records an error word and every CTA returns.
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

constexpr int kFusedThreads = 128;                              // 4 warps: one item or one algebra claim
constexpr int kFusedMinBlocks = 3;                              // CTAs per SM (168 registers)
constexpr unsigned long long kFusedWaitNs = 2000000000ull;      // 2 s per wait, then an error
constexpr size_t kFusedStageBytes = (size_t)kNumDerivs * kStageW * sizeof(float);  // per warp
constexpr size_t kFusedSmemBytes = 4 * kFusedStageBytes;        // 70,656 B (derivative buffers alias it)
static_assert(4 * kPlane * sizeof(double) + 2 * kDxRows * kTileX * sizeof(double) +
                      (kHalo + 1) * kDerivThreads * sizeof(double) <= kFusedSmemBytes,
              "the derivative item's buffers fit in the algebra staging area");
static_assert(kFusedThreads == kDerivThreads, "one CTA shape for both roles");

// Device words of one evaluation, zeroed before the launch:
//   [0] next item, [1] algebra hint, [2] error (1: a wait timed out), [3] unused,
//   done[ntiles] (items finished), claimed[ntiles] (planes whose algebra is claimed),
//   used[ntiles] (planes whose algebra is finished), gen[nring] (slot s is free for
//   tile-slab T when gen[s] == T / nring)
struct FusedArgs {
  DerivArgs d;        // state, blocks; dscr/koscr = the ring (MIXED: float)
  AlgebraArgs a;      // state, RHS or RK4 stage, parameters
  const FusedTileDev* tiles;
  int32_t ntiles, nring;
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
constexpr int kFusedPlanes = 2;  // planes of one algebra claim

// Warp 0: the next unit of work for this CTA (see the scheduling note above).  The
// CTA's held item (`pending`, -1 for none) survives between calls.  Returns the role;
// *idx is the item or the tile-slab, *p0 / *np the planes of an algebra claim.
__device__ __forceinline__ int fused_schedule(const FusedArgs& f, int& pending, int* idx, int* p0, int* np) {
  const int lane = threadIdx.x & 31;
  int* const next_item = f.sync + 0;
  int* const hint = f.sync + 1;
  int* const err = f.sync + 2;
  const int* const done = f.sync + 4;
  int* const claimed = f.sync + 4 + f.ntiles;
  const int* const gen = f.sync + 4 + 3 * f.ntiles;
  const int nitems = f.ntiles * kNumVars;
  unsigned long long t0 = 0;
  unsigned sleep = 32;
  for (;;) {
    if (ld_relaxed(err)) return FR_EXIT;
    // algebra: the 32 tile-slabs from the hint, one per lane
    const int h = ld_relaxed(hint);
    const int T = h + lane;
    const bool inwin = T < f.ntiles && lane < f.nring;
    int nz = 0, dn = 0, cl = 0;
    if (inwin) {
      nz = f.tiles[T].nz;
      dn = ld_relaxed(done + T);
      cl = ld_relaxed(claimed + T);
    }
    const bool ready = inwin && dn == kNumVars && cl < nz;
    const unsigned exhausted = __ballot_sync(0xffffffffu, inwin && dn == kNumVars && cl >= nz);
    const int adv = exhausted == 0xffffffffu ? 32 : __ffs(~exhausted) - 1;  // leading fully claimed tile-slabs
    if (adv > 0 && lane == 0) atomicMax(hint, h + adv);
    unsigned rmask = __ballot_sync(0xffffffffu, ready);
    while (rmask) {
      const int l = __ffs(rmask) - 1;
      int c = 0;
      if (lane == l) c = atomicAdd(claimed + T, kFusedPlanes);
      c = __shfl_sync(0xffffffffu, c, l);
      const int nzl = __shfl_sync(0xffffffffu, nz, l);
      if (c < nzl) {
        __threadfence();  // the tile-slab's slots are read after its done count
        *idx = h + l;
        *p0 = c;
        *np = min(kFusedPlanes, nzl - c);
        return FR_GROUP;
      }
      rmask &= rmask - 1;
    }
    // an item: the one this CTA holds, or the next one
    if (pending < 0 && ld_relaxed(next_item) < nitems) {
      int d = 0;
      if (lane == 0) d = atomicAdd(next_item, 1);
      d = __shfl_sync(0xffffffffu, d, 0);
      if (d < nitems) pending = d;
    }
    if (pending >= 0) {
      const int Tp = pending / kNumVars;
      if (ld_relaxed(gen + Tp % f.nring) == Tp / f.nring) {
        __threadfence();  // the slot's previous readers are done before it is rewritten
        *idx = pending;
        pending = -1;
        return FR_ITEM;
      }
    } else if (h >= f.ntiles) {
      return FR_EXIT;  // every item and every plane's algebra is claimed
    }
    // nothing can be claimed now: the work that unblocks it is running on other CTAs
    const unsigned long long now = global_ns();
    if (t0 == 0) {
      t0 = now;
    } else if (now - t0 > kFusedWaitNs) {
      if (lane == 0) atomicExch(err, 1);
      return FR_EXIT;
    }
    __nanosleep(sleep);
    sleep = min(sleep * 2, 512u);
  }
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
  __shared__ int s_role, s_idx, s_p0, s_np;
  double* s_plane = reinterpret_cast<double*>(smem);
  double* s_dxp = reinterpret_cast<double*>(smem + 4 * kPlane * sizeof(double));
  double* s_kq = s_dxp + 2 * kDxRows * kTileX;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* const done = f.sync + 4;
  int* const used = f.sync + 4 + 2 * f.ntiles;
  int* const gen = f.sync + 4 + 3 * f.ntiles;
  int pending = -1;  // warp 0: the item this CTA holds

  for (;;) {
    if (warp == 0) {
      int idx = 0, p0 = 0, np = 0;
      const int role = fused_schedule(f, pending, &idx, &p0, &np);
      if (lane == 0) {
        s_role = role;
        s_idx = idx;
        s_p0 = p0;
        s_np = np;
      }
    }
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
      const int T = idx, pz0 = s_p0, npl = s_np;
      const FusedTileDev ft = f.tiles[T];
      const BlockDev& B = f.a.blocks[ft.block];
      const int tx = lane & 15, ty = 2 * warp + (lane >> 4);
      const bool any = 2 * warp < ft.ey;
      const bool valid = tx < ft.ex && ty < ft.ey;
      float* sd = reinterpret_cast<float*>(smem + warp * kFusedStageBytes);
      for (int z = pz0; any && z < pz0 + npl; ++z) {
        const int run = (T % f.nring) * (kFusedSlotPts / 32) + z * 4 + warp;  // 32-point run in the ring
        const float* gd = static_cast<const float*>(f.d.dscr) + (size_t)run * kNumDerivs * 32;
        const float* gk = static_cast<const float*>(f.d.koscr) + (size_t)run * kNumVars * 32;
        const int i = 3 + ft.i0 + tx, j = 3 + ft.j0 + ty, k = 3 + ft.k0 + z;
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
        __syncwarp();  // every lane is done with the previous plane's copy
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
        if (atomicAdd(used + T, npl) + npl == ft.nz) {
          __threadfence();
          atomicExch(gen + T % f.nring, T / f.nring + 1);  // the slot is free for T + nring
        }
      }
    }
    __syncthreads();  // s_role and the shared buffers are free for the next unit
  }
}

}  // namespace b200bssn
