// NaN/Inf guard over a plan's interior points: one thread per interior point (the
// plan's algebra ranges), each scanning the requested arrays and recording the
// smallest element index that holds a non-finite value.  A time-step loop calls it
// between steps to stop on a blown-up state before the next launch.
#include <cuda_runtime.h>

#include <cstring>

#include "b200bssn.h"
#include "plan_internal.h"
#include "plan_types.h"

using namespace b200bssn;
using b200bssn::host::fail_cuda;

#define CK B200BSSN_CK

namespace {

struct GuardArgs {
  const double* a[kNumVars];
  int32_t narrays;
  const BlockDev* blocks;
  const UnitDev* units;
  const RangeDev* ranges;
  unsigned long long* first_bad;
};

__global__ void __launch_bounds__(kAlgebraThreads) finite_guard_kernel(const __grid_constant__ GuardArgs g) {
  const RangeDev rg = g.ranges[blockIdx.x];
  if ((int)threadIdx.x >= rg.count) return;
  const UnitDev un = g.units[rg.unit];
  const BlockDev& B = g.blocks[un.block];
  const int nx = B.sz[0], ny = B.sz[1];
  const int I0 = nx - 6, I1 = ny - 6;
  const int lpu = rg.start + threadIdx.x;
  const int lx = lpu % I0, rr = lpu / I0, ly = rr % I1, lz = rr / I1;
  const unsigned long long pp =
      B.offset + (lx + 3) + (unsigned long long)nx * ((ly + 3) + (unsigned long long)ny * (lz + 3 + un.k0));
  bool bad = false;
  for (int v = 0; v < g.narrays; ++v) bad |= !isfinite(__ldg(g.a[v] + pp));
  if (bad) atomicMin(g.first_bad, pp);
}

}  // namespace

extern "C" {

int b200bssn_check_finite(b200bssn_plan* P, const double* const* arrays, uint32_t narrays,
                          uint64_t* first_bad, void* stream) {
  b200bssn::host::NvtxRange nvtx_("b200bssn_check_finite");
  if (!P || !arrays || narrays == 0 || narrays > (uint32_t)kNumVars) return B200BSSN_ERR_INVALID_ARGUMENT;
  for (uint32_t v = 0; v < narrays; ++v)
    if (!arrays[v]) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = P->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  if (!P->d_guard) CK(ctx, cudaMalloc((void**)&P->d_guard, sizeof(unsigned long long)));
  GuardArgs g;
  std::memset(&g, 0, sizeof(g));
  for (uint32_t v = 0; v < narrays; ++v) g.a[v] = arrays[v];
  g.narrays = (int32_t)narrays;
  g.blocks = P->d_blocks;
  g.units = P->d_units;
  g.ranges = P->d_ranges;
  g.first_bad = P->d_guard;
  CK(ctx, cudaMemsetAsync(P->d_guard, 0xff, sizeof(unsigned long long), s));
  finite_guard_kernel<<<(unsigned)P->ranges.size(), kAlgebraThreads, 0, s>>>(g);
  CK(ctx, cudaGetLastError());
  unsigned long long h = 0;
  CK(ctx, cudaMemcpyAsync(&h, P->d_guard, sizeof(h), cudaMemcpyDeviceToHost, s));
  CK(ctx, cudaStreamSynchronize(s));
  if (first_bad) *first_bad = h;
  return h == ~0ull ? B200BSSN_OK : B200BSSN_ERR_NONFINITE;
}

}  // extern "C"
