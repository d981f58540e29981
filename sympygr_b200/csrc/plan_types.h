// Work-plan descriptors shared by the host planner and the kernels.
//
// A plan covers a list of octree blocks.  Each block's interior (sz-6)^3 is cut
// into z-slabs ("units", by default at most 48 planes); a unit's points are numbered
// compactly, x fastest:  lp = (i-3) + I0*((j-3) + I1*(k-3-k0)).  Units are packed
// into chunks whose total point count fits the derivative scratch; each chunk is
// evaluated by one derivative launch (one CTA per 16x8 column tile of a unit,
// streaming along z through all variables) followed by one algebra launch (one
// CTA per run of consecutive points of a unit).
#pragma once
#include <stdint.h>

namespace b200bssn {

constexpr int kNumVars = 24;
constexpr int kNumDerivs = 138;  // algebra inputs: 72 first + 66 second derivatives
constexpr int kTileX = 16, kTileY = 8;
constexpr int kTileZ = 48;       // default z-slab depth (measured best on the 3000-block batch)
constexpr int kHalo = 4;         // closure rows reach four points inward (z queue: 4 each side)
constexpr int kDerivThreads = 128;
constexpr int kAlgebraThreads = 128;

struct BlockDev {
  uint64_t offset;   // element offset in every variable array
  int32_t sz[3];
  uint32_t bflag;
  double pmin[3];    // ghost-inclusive corner
  double h[3];       // (pmax - pmin)/(sz - 1), computed on the host as bssnrhs does
};

struct UnitDev {
  int32_t block;
  int32_t k0;        // first interior plane of the slab (0-based interior index)
  int32_t nz;        // planes in the slab (<= kTileZ)
  int32_t pad;
  int64_t sbase;     // first scratch point of the unit within its chunk
};

struct TileDev {
  int32_t unit;
  int16_t i0, j0;    // interior-relative origin of the x-y tile
  int16_t ex, ey;    // extents (<= kTileX, kTileY)
};

// One tile-slab of the one-pass kernel: a 16x8 column tile of a block over a z-slab
// of at most kFusedSlab interior planes.
struct FusedTileDev {
  int32_t block;
  int16_t i0, j0;     // interior-relative x-y origin of the tile
  int16_t ex, ey;     // extents (<= kTileX, kTileY)
  int16_t k0, nz;     // interior-relative first plane and planes (<= kFusedSlab)
  int32_t pad;
};
constexpr int kFusedSlab = 24;                               // max interior planes per tile-slab
constexpr int kFusedSlotPts = kTileX * kTileY * kFusedSlab;  // 3072 points per ring slot
constexpr int kFusedRingDefault = 128;                       // slots: 256 MB in MIXED

struct RangeDev {
  int32_t unit;
  int32_t start;     // first compact point index within the unit
  int32_t count;     // <= kAlgebraThreads
};

// Classic RK4 stage update fused into the algebra kernel's epilogue.  With k the
// right-hand side at a point (in FP64, KO included) and u^n the state at the start
// of the step:
//   RK_FIRST   acc  = w k          next = u^n + c k      (stage 1)
//   RK_MIDDLE  acc += w k          next = u^n + c k      (stages 2, 3)
//   RK_LAST    u^n  = u^n + acc + w k                     (stage 4)
// with w = dt/6, dt/3, dt/3, dt/6 and c = dt/2, dt/2, dt.  Every array is read and
// written at the thread's own point only, so the kernel's inputs (the stage state
// `u`, read at the point and by the derivative kernel) never alias its outputs.
enum RkMode : int32_t { RK_NONE = 0, RK_FIRST = 1, RK_MIDDLE = 2, RK_LAST = 3 };

struct RkStage {
  int32_t mode;
  double w, c;
  double* acc[kNumVars];
  double* next[kNumVars];
  double* base[kNumVars];  // u^n: read in every stage, written in RK_LAST
};

// Scratch layout (derivative slots and KO sums): blocks of 32 consecutive points
// (chunk-relative index lp), each block holding its NS slots one after another --
// value (slot s, point lp) at ((lp / 32) * NS + s) * 32 + lp % 32.  A 32-point task
// of the algebra kernel then reads one contiguous run of NS * 32 values instead of
// NS columns far apart (a copy of that shape reaches the full HBM read rate; 138
// scattered 128-byte pieces per task reach about two thirds of it).
template <int NS>
__device__ __forceinline__ int scr_index(int s, int lp) {
  return ((lp >> 5) * NS + s) * 32 + (lp & 31);
}
__device__ __forceinline__ int scr_index(int ns, int s, int lp) {
  return ((lp >> 5) * ns + s) * 32 + (lp & 31);
}

}  // namespace b200bssn
