// b200bssn_rhs_noalloc: the right-hand side of one block with no device
// allocation at all.
//
// Who needs this: a solver framework that hands the whole GPU memory to its own
// pool allocator at start-up (so a library cudaMalloc would fail or fragment that
// pool), and a time-step loop that must not call cudaMalloc/cudaFree because they
// can synchronise the whole device.  Such callers own the input and output arrays;
// the only other memory this path needs -- the derivative scratch and the work
// descriptors -- lives in one fixed array below, reserved when the library is
// loaded and held by every GPU that loads it until the process exits.
//
// Limits and sharing:
//  * at most kNoallocMaxPoints interior points per call (a block with a 32^3
//    interior, i.e. 38^3 padded, is the largest cube that fits); larger blocks
//    are rejected with B200BSSN_ERR_SIZE_LIMIT before anything is launched;
//  * every call on a device uses the same array, which keeps whatever the last
//    call left in it.  Each call rewrites every word it later reads (descriptors
//    first, then every derivative slot of every interior point), so nothing has
//    to start at zero -- but two calls whose work overlaps on the GPU (different
//    streams, or host threads racing) overwrite each other's scratch and give
//    wrong results.  Serialise calls per device;
//  * the first call on each device looks up the array's device address with
//    cudaGetSymbolAddress, sets the derivative kernel's shared-memory limit and
//    reads its occupancy, with that device current; make that first call before any
//    stream capture.  The address is kept for the life of the process, so calls after
//    a cudaDeviceReset of that device (which reloads the library's device code at a
//    new address) are not supported.
//
// The derivative kernel here is the combined one over all 24 variables
// (bssn_derivs_kernel), which only this entry point launches; the plans use the two
// per-kind kernels.
#include <cuda_runtime.h>

#include <cstring>

#include <mutex>

#include "b200bssn.h"
#include "rhs_kernels.cuh"

using namespace b200bssn;

namespace {

constexpr int64_t kNoallocMaxPoints = B200BSSN_NOALLOC_MAX_POINTS;
constexpr int kNoallocMaxUnits = 1024;
constexpr int kNoallocMaxTiles = 4096;
constexpr int kNoallocMaxRanges = 2048;
constexpr int kMaxDevices = 64;
constexpr int kNoallocSlab = 48;  // z-slab depth of this path's work units

// byte layout of the fixed array (each part 256-byte aligned)
constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffCounter = 0;
constexpr size_t kOffBlock = kOffCounter + 256;
constexpr size_t kOffUnits = kOffBlock + al256(sizeof(BlockDev));
constexpr size_t kOffTiles = kOffUnits + al256(sizeof(UnitDev) * kNoallocMaxUnits);
constexpr size_t kOffRanges = kOffTiles + al256(sizeof(TileDev) * kNoallocMaxTiles);
constexpr size_t kOffDeriv = kOffRanges + al256(sizeof(RangeDev) * kNoallocMaxRanges);
constexpr size_t kOffKo = kOffDeriv + al256(sizeof(double) * kNumDerivs * kNoallocMaxPoints);
// + 256: the algebra kernel's L2 prefetch of a slot run rounds its size up to 16 bytes
constexpr size_t kNoallocBytes = kOffKo + al256(sizeof(double) * kNumVars * kNoallocMaxPoints) + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// Per-device address of g_noalloc_scratch (host-side handle -> device address) and
// the resident CTA count of the persistent derivative kernel, per precision.
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};
int g_deriv_grid[kMaxDevices][2] = {};  // [dev][0: FP64, 1: MIXED]

int setup_device(int dev, void** addr, int* grid64, int* grid32) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_addr[dev]) {
    *addr = g_scratch_addr[dev];
    *grid64 = g_deriv_grid[dev][0];
    *grid32 = g_deriv_grid[dev][1];
    return B200BSSN_OK;
  }
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
    cudaGetLastError();
    return B200BSSN_ERR_CUDA;
  }
  if (cudaFuncSetAttribute(bssn_derivs_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kDerivSmemBytes) != cudaSuccess ||
      cudaFuncSetAttribute(bssn_derivs_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kDerivSmemBytes) != cudaSuccess) {
    cudaGetLastError();
    return B200BSSN_ERR_CUDA;
  }
  // the derivative kernel is persistent (each CTA pulls items from the work counter),
  // so its grid is the CTAs that fit on the GPU at once, as the plans size it
  int sms = 0, occ64 = 0, occ32 = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ64, bssn_derivs_kernel<double>, kDerivThreads,
                                                    kDerivSmemBytes) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ32, bssn_derivs_kernel<float>, kDerivThreads,
                                                    kDerivSmemBytes) != cudaSuccess ||
      sms <= 0 || occ64 <= 0 || occ32 <= 0) {
    cudaGetLastError();
    return B200BSSN_ERR_CUDA;
  }
  g_deriv_grid[dev][0] = sms * occ64;
  g_deriv_grid[dev][1] = sms * occ32;
  g_scratch_addr[dev] = p;
  *addr = p;
  *grid64 = g_deriv_grid[dev][0];
  *grid32 = g_deriv_grid[dev][1];
  return B200BSSN_OK;
}

// Writes the work descriptors of one block (z-slab units of kNoallocSlab planes, x-y
// tiles, runs of kAlgebraThreads points) -- the layout b200bssn_plan_create
// builds on the host -- straight into the fixed array.
__global__ void noalloc_describe(BlockDev blk, BlockDev* blk_out, int* counter, UnitDev* units,
                                 TileDev* tiles, RangeDev* ranges, int n_units, int tiles_x,
                                 int tiles_y, int ranges_per_unit_max) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *blk_out = blk;
    *counter = 0;  // work counter of the derivative kernel
  }
  const int I0 = blk.sz[0] - 6, I1 = blk.sz[1] - 6, I2 = blk.sz[2] - 6;
  const int tiles_per_unit = tiles_x * tiles_y;
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < n_units; u += gridDim.x * blockDim.x) {
    UnitDev d;
    d.block = 0;
    d.k0 = u * kNoallocSlab;
    d.nz = min(kNoallocSlab, I2 - d.k0);
    d.pad = 0;
    d.sbase = (int64_t)I0 * I1 * d.k0;
    units[u] = d;
    const int np = I0 * I1 * d.nz;
    for (int r = 0; r < ranges_per_unit_max; ++r) {
      RangeDev g;
      g.unit = u;
      g.start = r * kAlgebraThreads;
      g.count = max(0, min(kAlgebraThreads, np - g.start));
      ranges[u * ranges_per_unit_max + r] = g;
    }
    for (int t = 0; t < tiles_per_unit; ++t) {
      TileDev td;
      td.unit = u;
      const int tx = t % tiles_x, ty = t / tiles_x;
      td.i0 = (int16_t)(tx * kTileX);
      td.j0 = (int16_t)(ty * kTileY);
      td.ex = (int16_t)min(kTileX, I0 - tx * kTileX);
      td.ey = (int16_t)min(kTileY, I1 - ty * kTileY);
      tiles[u * tiles_per_unit + t] = td;
    }
  }
}

}  // namespace

extern "C" int b200bssn_rhs_noalloc(double* const* rhs_dev, const double* const* u_dev,
                                    const b200bssn_block* block, const b200bssn_params* prm,
                                    void* stream) {
  if (!rhs_dev || !u_dev || !block || !prm) return B200BSSN_ERR_INVALID_ARGUMENT;
  if (prm->precision != B200BSSN_FP64 && prm->precision != B200BSSN_MIXED)
    return B200BSSN_ERR_INVALID_ARGUMENT;
  for (int v = 0; v < kNumVars; ++v)
    if (!rhs_dev[v] || !u_dev[v]) return B200BSSN_ERR_INVALID_ARGUMENT;
  for (int a = 0; a < 3; ++a) {
    if (block->sz[a] < 13) return B200BSSN_ERR_BLOCK_TOO_SMALL;
    if (!(block->pmax[a] > block->pmin[a])) return B200BSSN_ERR_INVALID_ARGUMENT;
  }
  if (block->bflag >> 6) return B200BSSN_ERR_INVALID_ARGUMENT;
  const int64_t I0 = block->sz[0] - 6, I1 = block->sz[1] - 6, I2 = block->sz[2] - 6;
  const int64_t npts = I0 * I1 * I2;
  const int64_t n_units = (I2 + kNoallocSlab - 1) / kNoallocSlab;
  const int64_t tiles_x = (I0 + kTileX - 1) / kTileX, tiles_y = (I1 + kTileY - 1) / kTileY;
  const int64_t rpu = (I0 * I1 * kNoallocSlab + kAlgebraThreads - 1) / kAlgebraThreads;
  if (npts > kNoallocMaxPoints || n_units > kNoallocMaxUnits ||
      n_units * tiles_x * tiles_y > kNoallocMaxTiles || n_units * rpu > kNoallocMaxRanges)
    return B200BSSN_ERR_SIZE_LIMIT;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return B200BSSN_ERR_NO_DEVICE;
  }
  void* base = nullptr;
  int grid64 = 0, grid32 = 0;
  int rc = setup_device(dev, &base, &grid64, &grid32);
  if (rc != B200BSSN_OK) return rc;
  char* b = static_cast<char*>(base);
  UnitDev* units = reinterpret_cast<UnitDev*>(b + kOffUnits);
  TileDev* tiles = reinterpret_cast<TileDev*>(b + kOffTiles);
  RangeDev* ranges = reinterpret_cast<RangeDev*>(b + kOffRanges);
  BlockDev* bd = reinterpret_cast<BlockDev*>(b + kOffBlock);

  BlockDev blk;
  blk.offset = block->offset;
  blk.bflag = block->bflag;
  for (int a = 0; a < 3; ++a) {
    blk.sz[a] = (int32_t)block->sz[a];
    blk.pmin[a] = block->pmin[a];
    blk.h[a] = (block->pmax[a] - block->pmin[a]) / (block->sz[a] - 1);  // rhs.cpp:144-146
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the block descriptor travels as a kernel argument and the kernel stores it,
  // so no host-to-device copy is needed either
  int* counter = reinterpret_cast<int*>(b + kOffCounter);
  noalloc_describe<<<(int)((n_units + 127) / 128), 128, 0, s>>>(blk, bd, counter, units, tiles,
                                                                ranges, (int)n_units, (int)tiles_x,
                                                                (int)tiles_y, (int)rpu);

  DerivArgs da;
  AlgebraArgs aa;
  std::memset(&da, 0, sizeof(da));
  std::memset(&aa, 0, sizeof(aa));  // aa.rk.mode = RK_NONE: store the RHS
  for (int v = 0; v < kNumVars; ++v) {
    da.u[v] = u_dev[v];
    aa.u[v] = u_dev[v];
    aa.rhs[v] = rhs_dev[v];
  }
  da.blocks = aa.blocks = bd;
  da.units = aa.units = units;
  da.tiles = tiles;
  aa.ranges = ranges;
  da.dscr = b + kOffDeriv;
  aa.dscr = b + kOffDeriv;
  da.koscr = b + kOffKo;
  aa.koscr = da.koscr;
  da.cap = aa.cap = (int32_t)kNoallocMaxPoints;
  da.tile_base = 0;
  da.tile_count = (int32_t)(n_units * tiles_x * tiles_y);
  da.counter = counter;
  aa.range_base = 0;
  aa.prm64 = {(double)prm->lambda[0], (double)prm->lambda[1], (double)prm->lambda[2],
              (double)prm->lambda[3], prm->lambda_f[0], prm->lambda_f[1]};
  aa.prm32 = {(float)prm->lambda[0], (float)prm->lambda[1], (float)prm->lambda[2],
              (float)prm->lambda[3], (float)prm->lambda_f[0], (float)prm->lambda_f[1]};
  aa.eta_const = prm->eta_const;
  aa.eta_r0 = prm->eta_r0;
  aa.eta_damping_exp = prm->eta_damping_exp;
  aa.ko_sigma = prm->ko_sigma;

  const int64_t items = n_units * tiles_x * tiles_y * kNumVars;
  const int64_t gmax = prm->precision == B200BSSN_MIXED ? grid32 : grid64;
  const dim3 g1((unsigned)(items < gmax ? items : gmax), 1);
  const unsigned g2 = (unsigned)(n_units * rpu);  // runs past a unit's end have count 0
  if (prm->precision == B200BSSN_MIXED) {
    bssn_derivs_kernel<float><<<g1, kDerivThreads, kDerivSmemBytes, s>>>(da);
    bssn_algebra_kernel<float, float><<<g2, kAlgebraThreads, 0, s>>>(aa);
  } else {
    bssn_derivs_kernel<double><<<g1, kDerivThreads, kDerivSmemBytes, s>>>(da);
    bssn_algebra_kernel<double, double><<<g2, kAlgebraThreads, 0, s>>>(aa);
  }
  if (cudaGetLastError() != cudaSuccess) return B200BSSN_ERR_CUDA;
  return B200BSSN_OK;
}
