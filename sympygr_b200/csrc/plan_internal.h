// Internal host-side state of libb200bssn shared by its translation units: the
// context and plan objects behind the opaque handles of include/b200bssn.h, and
// the plan launcher the right-hand-side, constraint and RK4 entry points share.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <string>
#include <vector>

#include "b200bssn.h"
#include "plan_types.h"

namespace b200bssn {
struct ConstraintArgs;
}  // namespace b200bssn

using b200bssn::BlockDev;
using b200bssn::RangeDev;
using b200bssn::TileDev;
using b200bssn::UnitDev;

struct b200bssn_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // derivative and algebra streams of the chunk pipeline (see launch_plan), and
  // the upload / download streams of the pipelined host path
  cudaStream_t s_deriv = nullptr, s_alg = nullptr, s_h2d = nullptr, s_d2h = nullptr;
  std::string last_error;
  // single-block drop-in path
  double* blk_u = nullptr;    // [24][npad]
  double* blk_rhs = nullptr;  // [24][npad]
  size_t blk_cap = 0;         // npad capacity
  b200bssn_plan* blk_plan = nullptr;
  uint32_t blk_sz[3] = {0, 0, 0};
  uint32_t blk_precision = 0xffffffffu;
  // pinned host staging of the block's state (upload) and results (download), and
  // one event per variable marking its download done
  double* blk_pin = nullptr;
  size_t blk_pin_cap = 0;  // doubles
  cudaEvent_t blk_ev[b200bssn::kNumVars] = {};
};

struct ChunkRec {
  int32_t tile_begin, tile_count;
  int32_t range_begin, range_count;
  int64_t points;
};

struct b200bssn_plan {
  b200bssn_ctx* ctx = nullptr;
  uint32_t precision = 0;
  bool advective = false;  // upwind mode: 72 more scratch slots (advective derivatives)
  std::vector<BlockDev> blocks;
  std::vector<UnitDev> units;
  std::vector<TileDev> tiles;
  std::vector<RangeDev> ranges;
  std::vector<ChunkRec> chunks;
  uint64_t points = 0;
  int64_t cap = 0;
  uint64_t span_lo = 0, span_hi = 0;  // element range touched in the variable arrays
  // device
  void* desc = nullptr;  // blocks | units | tiles | ranges
  BlockDev* d_blocks = nullptr;
  UnitDev* d_units = nullptr;
  TileDev* d_tiles = nullptr;
  RangeDev* d_ranges = nullptr;
  // derivative scratch: two buffers when the plan has more than one chunk, so the
  // derivative kernel of chunk c+1 can run while the algebra kernel of chunk c reads
  void* dscr[2] = {nullptr, nullptr};
  void* koscr[2] = {nullptr, nullptr};  // KO sums, stored like the slots (double or float)
  std::vector<cudaEvent_t> ev_deriv, ev_alg;  // per chunk: derivative / algebra done
  cudaEvent_t ev_fork = nullptr;
  int* d_counters = nullptr;  // per chunk: work counter of the derivative kernel
  unsigned long long* d_guard = nullptr;  // finiteness check result (allocated on first use)
  // pipelined host path: element ranges [part[c], part[c+1]) partition the span, one
  // per chunk, when chunks hold whole blocks in increasing offset order
  bool host_pipeline = false;
  std::vector<uint64_t> part;
  std::vector<std::vector<int32_t>> chunk_blocks;  // per chunk: its blocks (host pipeline)
  std::vector<cudaEvent_t> ev_in;  // per chunk: upload done
  int tile_y = b200bssn::kTileY;      // tile height of the derivative kernels (4, 8 or 16)
  int deriv_regs = 0;                 // register split variant of the derivative kernels
  const void* kind_fn[2] = {nullptr, nullptr};  // the derivative kind kernels (without / with DD)
  int deriv_threads = 128;            // threads per derivative CTA
  int deriv_grid[2] = {0, 0};  // resident CTAs of the two persistent derivative kernels
  int alg_grid = 0;           // resident CTAs of the persistent staged algebra kernel (MIXED)
  // one-pass path (MIXED, centred advection): tile-slabs in launch order, the
  // per-evaluation sync words and the scratch ring
  bool single_pass = false;
  int32_t nring = 0, fused_grid = 0;
  std::vector<b200bssn::FusedTileDev> ftiles;
  void* fdesc = nullptr;
  b200bssn::FusedTileDev* d_ftiles = nullptr;
  int* d_fsync = nullptr;
  size_t fsync_words = 0;
  void* fring_d = nullptr;  // nring * kFusedSlotPts points x 138 slots (float)
  void* fring_k = nullptr;  // nring * kFusedSlotPts points x 24 KO sums (float)
  // host-batch staging (allocated on first host call)
  double* st_u = nullptr;
  double* st_rhs = nullptr;
  uint64_t st_len = 0;
  // st_rhs holds zeros wherever no kernel writes (ghost points, gaps between blocks):
  // the kernels write interior points only, so one clearing lasts until a
  // ghost-preserving call puts the caller's values there
  bool st_rhs_zeroed = false;
};

namespace b200bssn {
namespace host {

// NVTX range around an entry point (shows in Nsight Systems timelines; a no-op
// unless a tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Records the CUDA error text on the context and maps it to a status code.
int fail_cuda(b200bssn_ctx* ctx, cudaError_t e, const char* what);

bool params_ok(const b200bssn_params* p);

// Enqueues one evaluation of the plan on stream `s` (see b200bssn.cu).  `rk`
// non-null: the algebra kernel applies that RK4 stage update instead of storing
// the RHS; `ca` non-null: the constraint kernel replaces the algebra kernel.
int launch_plan(b200bssn_plan* P, double* const* rhs, const double* const* u,
                const b200bssn_params* prm, cudaStream_t s, cudaEvent_t* ev = nullptr,
                const ConstraintArgs* ca = nullptr, const RkStage* rk = nullptr);

}  // namespace host
}  // namespace b200bssn

#define B200BSSN_CK(ctx, call)                                                        \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) return ::b200bssn::host::fail_cuda(ctx, e_, #call);        \
  } while (0)
