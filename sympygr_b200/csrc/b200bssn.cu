// Host side of libb200bssn: contexts, work plans and the C ABI declared in
// include/b200bssn.h.  The kernels are in rhs_kernels.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "b200bssn.h"
#include "constraint_kernels.cuh"
#include "fused_kernel.cuh"
#include "plan_internal.h"
#include "rhs_kernels.cuh"

using namespace b200bssn;
using b200bssn::host::fail_cuda;
using b200bssn::host::launch_plan;
using b200bssn::host::params_ok;

int b200bssn::host::fail_cuda(b200bssn_ctx* ctx, cudaError_t e, const char* what) {
  if (ctx) {
    ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
  }
  return e == cudaErrorMemoryAllocation ? B200BSSN_ERR_OUT_OF_MEMORY : B200BSSN_ERR_CUDA;
}

bool b200bssn::host::params_ok(const b200bssn_params* p) {
  return p && (p->precision == B200BSSN_FP64 || p->precision == B200BSSN_MIXED) &&
         (p->ghost_policy == B200BSSN_GHOSTS_PRESERVE || p->ghost_policy == B200BSSN_GHOSTS_ZERO);
}

#define CK B200BSSN_CK

namespace {

constexpr int64_t kDefaultChunkPoints = int64_t(1) << 23;
// scratch slots are addressed with 32-bit offsets: slots * cap < 2^31 (slots: 138, or
// 210 in the upwind mode)
constexpr int64_t max_chunk_points(int slots) { return (int64_t(1) << 31) / (slots + 1) - 1; }

void make_args(const b200bssn_plan* P, double* const* rhs, const double* const* u,
               const b200bssn_params* prm, DerivArgs& da, AlgebraArgs& aa) {
  std::memset(&da, 0, sizeof(da));
  std::memset(&aa, 0, sizeof(aa));  // aa.rk.mode = RK_NONE: store the RHS
  for (int v = 0; v < kNumVars; ++v) {
    da.u[v] = u[v];
    aa.u[v] = u[v];
    aa.rhs[v] = rhs[v];
  }
  da.blocks = aa.blocks = P->d_blocks;
  da.units = aa.units = P->d_units;
  da.tiles = P->d_tiles;
  aa.ranges = P->d_ranges;
  da.cap = aa.cap = (int32_t)P->cap;
  aa.prm64 = {(double)prm->lambda[0], (double)prm->lambda[1], (double)prm->lambda[2],
              (double)prm->lambda[3], prm->lambda_f[0], prm->lambda_f[1]};
  aa.prm32 = {(float)prm->lambda[0], (float)prm->lambda[1], (float)prm->lambda[2],
              (float)prm->lambda[3], (float)prm->lambda_f[0], (float)prm->lambda_f[1]};
  aa.eta_const = prm->eta_const;
  aa.eta_r0 = prm->eta_r0;
  aa.eta_damping_exp = prm->eta_damping_exp;
  aa.ko_sigma = prm->ko_sigma;
}

// The derivative kind kernels built for each plan knob: tile height 4, 8 or 16 with the
// default register split, and 16x8 tiles with one CTA per SM more or fewer (the upwind
// mode only with the defaults).  Returns the kernel, or nullptr if not built.
template <typename ST, bool ADV, int TY, int REGV>
const void* kind_ptr(bool dd) {
  return dd ? (const void*)bssn_derivs_kind_kernel<ST, true, ADV, TY, REGV>
            : (const void*)bssn_derivs_kind_kernel<ST, false, ADV, TY, REGV>;
}
const void* kind_kernel(bool mixed, bool adv, bool dd, int ty, int regv) {
  if (adv) {
    if (ty != kTileY || regv != 0) return nullptr;
    return mixed ? kind_ptr<float, true, kTileY, 0>(dd) : kind_ptr<double, true, kTileY, 0>(dd);
  }
#define B200BSSN_KIND(TYV, RV) \
  if (ty == TYV && regv == RV) return mixed ? kind_ptr<float, false, TYV, RV>(dd) : kind_ptr<double, false, TYV, RV>(dd);
  B200BSSN_KIND(8, 0)
  B200BSSN_KIND(8, 1)
  B200BSSN_KIND(8, 2)
  B200BSSN_KIND(4, 0)
  B200BSSN_KIND(16, 0)
#undef B200BSSN_KIND
  return nullptr;
}

// The derivative stage of one chunk: the kernels over the variables without and with
// second derivatives, each with its own work counter.
int launch_derivs(b200bssn_plan* P, DerivArgs dn, DerivArgs dd, int gn, int gd, cudaStream_t s) {
  void* an[] = {&dn};
  void* ad[] = {&dd};
  const dim3 block((unsigned)P->deriv_threads);
  CK(P->ctx, cudaLaunchKernel(P->kind_fn[0], dim3((unsigned)gn), block, an, 0, s));
  CK(P->ctx, cudaLaunchKernel(P->kind_fn[1], dim3((unsigned)gd), block, ad, 0, s));
  return B200BSSN_OK;
}

// The staged algebra kernel for the RK mode of `aa` (RK_NONE: store the RHS).
template <typename ST, bool ADV>
void launch_algebra(const AlgebraArgs& aa, unsigned grid, int ntasks, cudaStream_t s) {
  using Cfg = StageCfg<ST, ADV>;
  switch (aa.rk.mode) {
    case RK_FIRST:
      bssn_algebra_staged_kernel<ST, RK_FIRST, ADV><<<grid, Cfg::kThreads, Cfg::kSmemBytes, s>>>(aa, ntasks);
      break;
    case RK_MIDDLE:
      bssn_algebra_staged_kernel<ST, RK_MIDDLE, ADV><<<grid, Cfg::kThreads, Cfg::kSmemBytes, s>>>(aa, ntasks);
      break;
    case RK_LAST:
      bssn_algebra_staged_kernel<ST, RK_LAST, ADV><<<grid, Cfg::kThreads, Cfg::kSmemBytes, s>>>(aa, ntasks);
      break;
    default:
      bssn_algebra_staged_kernel<ST, RK_NONE, ADV><<<grid, Cfg::kThreads, Cfg::kSmemBytes, s>>>(aa, ntasks);
      break;
  }
}

template <typename ST, bool ADV>
int set_stage_attributes(b200bssn_ctx* ctx) {
  const int bytes = (int)StageCfg<ST, ADV>::kSmemBytes;
  CK(ctx, cudaFuncSetAttribute(bssn_algebra_staged_kernel<ST, RK_NONE, ADV>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CK(ctx, cudaFuncSetAttribute(bssn_algebra_staged_kernel<ST, RK_FIRST, ADV>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CK(ctx, cudaFuncSetAttribute(bssn_algebra_staged_kernel<ST, RK_MIDDLE, ADV>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CK(ctx, cudaFuncSetAttribute(bssn_algebra_staged_kernel<ST, RK_LAST, ADV>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return B200BSSN_OK;
}

// The two kernels of chunk ci: derivatives on s1, then on s2 the algebra or, with
// `ca` non-null, the constraint kernel (the caller orders s2 after s1 when they
// differ), scratch buffer `buf`.
int enqueue_chunk(b200bssn_plan* P, DerivArgs da, AlgebraArgs aa, size_t ci, int buf,
                  cudaStream_t s1, cudaStream_t s2, cudaEvent_t* ev,
                  const ConstraintArgs* ca = nullptr) {
  b200bssn_ctx* ctx = P->ctx;
  const ChunkRec& c = P->chunks[ci];
  const bool mixed = P->precision == B200BSSN_MIXED;
  da.tile_base = c.tile_begin;
  da.tile_count = c.tile_count;
  da.counter = P->d_counters + ci;
  aa.range_base = c.range_begin;
  da.dscr = P->dscr[buf];
  aa.dscr = P->dscr[buf];
  da.koscr = P->koscr[buf];
  aa.koscr = P->koscr[buf];
  if (ev) CK(ctx, cudaEventRecord(ev[4 * ci + 0], s1));
  {
    // the two derivative kernels (variables without, then with second derivatives),
    // each with its own work counter
    DerivArgs dn = da, dd = da;
    dn.counter = P->d_counters + 2 * ci;
    dd.counter = P->d_counters + 2 * ci + 1;
    const int gn = std::min(c.tile_count * kKindVars[0], P->deriv_grid[0]);
    const int gd = std::min(c.tile_count * kKindVars[1], P->deriv_grid[1]);
    const int rc = launch_derivs(P, dn, dd, gn, gd, s1);
    if (rc != B200BSSN_OK) return rc;
  }
  CK(ctx, cudaGetLastError());
  if (ev) CK(ctx, cudaEventRecord(ev[4 * ci + 1], s1));
  if (s1 != s2) {
    CK(ctx, cudaEventRecord(P->ev_deriv[ci], s1));
    CK(ctx, cudaStreamWaitEvent(s2, P->ev_deriv[ci], 0));
  }
  if (ev) CK(ctx, cudaEventRecord(ev[4 * ci + 2], s2));
  if (ca) {
    ConstraintArgs cc = *ca;
    cc.range_base = c.range_begin;
    cc.dscr = P->dscr[buf];
    if (mixed)
      bssn_constraints_kernel<float, float><<<c.range_count, kAlgebraThreads, 0, s2>>>(cc);
    else
      bssn_constraints_kernel<double, double><<<c.range_count, kAlgebraThreads, 0, s2>>>(cc);
  } else {
    // the staged persistent kernel: each warp takes 32-point tasks round-robin
    const int ntasks = c.range_count * (kAlgebraThreads / kStageW);
    const unsigned gs = (unsigned)std::max(1, std::min(P->alg_grid, ntasks));
    if (mixed)
      P->advective ? launch_algebra<float, true>(aa, gs, ntasks, s2)
                   : launch_algebra<float, false>(aa, gs, ntasks, s2);
    else
      P->advective ? launch_algebra<double, true>(aa, gs, ntasks, s2)
                   : launch_algebra<double, false>(aa, gs, ntasks, s2);
  }
  CK(ctx, cudaGetLastError());
  if (ev) CK(ctx, cudaEventRecord(ev[4 * ci + 3], s2));
  if (s1 != s2) CK(ctx, cudaEventRecord(P->ev_alg[ci], s2));
  return B200BSSN_OK;
}

// One evaluation as the one-pass kernel: zero the sync words, then one launch over
// every tile-slab of the plan.  With `ev` non-null, events ev[0], ev[1] around it.
int launch_single_pass(b200bssn_plan* P, const DerivArgs& da, const AlgebraArgs& aa, cudaStream_t s,
                       cudaEvent_t* ev) {
  b200bssn_ctx* ctx = P->ctx;
  FusedArgs f;
  std::memset(&f, 0, sizeof(f));
  f.d = da;
  f.a = aa;
  f.d.dscr = P->fring_d;
  f.d.koscr = P->fring_k;
  f.d.cap = P->nring * kFusedSlotPts;
  f.tiles = P->d_ftiles;
  f.ntiles = (int32_t)P->ftiles.size();
  f.nring = P->nring;
  f.sync = P->d_fsync;
  CK(ctx, cudaMemsetAsync(P->d_fsync, 0, P->fsync_words * sizeof(int), s));
  if (ev) CK(ctx, cudaEventRecord(ev[0], s));
  const unsigned grid = (unsigned)P->fused_grid;
  switch (aa.rk.mode) {
    case RK_FIRST:
      bssn_fused_kernel<RK_FIRST><<<grid, kFusedThreads, kFusedSmemBytes, s>>>(f);
      break;
    case RK_MIDDLE:
      bssn_fused_kernel<RK_MIDDLE><<<grid, kFusedThreads, kFusedSmemBytes, s>>>(f);
      break;
    case RK_LAST:
      bssn_fused_kernel<RK_LAST><<<grid, kFusedThreads, kFusedSmemBytes, s>>>(f);
      break;
    default:
      bssn_fused_kernel<RK_NONE><<<grid, kFusedThreads, kFusedSmemBytes, s>>>(f);
      break;
  }
  CK(ctx, cudaGetLastError());
  if (ev) CK(ctx, cudaEventRecord(ev[1], s));
  return B200BSSN_OK;
}

// Enqueues one evaluation of the plan.
//
// One-pass plans (MIXED, centred advection) run the right-hand side and the RK4
// stages as launch_single_pass; the constraints always take the two-pass kernels.
//
// With `ev` null and more than one chunk the chunks are pipelined over two
// internal streams: the derivative kernel of chunk c (stream s_deriv, scratch
// buffer c%2) runs while the algebra kernel of chunk c-1 (stream s_alg) is still
// reading the other buffer; event edges keep the order K1(c) -> K2(c) and
// K2(c-2) -> K1(c), and the caller's stream `s` forks into and joins from the
// two streams, so the whole evaluation is ordered on `s` (and can be captured
// into a CUDA graph from `s`).  With `ev` non-null (profiling) everything runs on
// `s` in order, with events ev[4c+0..3] around chunk c's two kernels.
//
// With `ca` non-null the second kernel of every chunk is the constraint kernel
// (`rhs` and `prm` are then only used to fill the unused algebra arguments); with
// `rk` non-null the algebra kernel applies that RK4 stage update (`rhs` unused).
}  // namespace

int b200bssn::host::launch_plan(b200bssn_plan* P, double* const* rhs, const double* const* u,
                                const b200bssn_params* prm, cudaStream_t s, cudaEvent_t* ev,
                                const ConstraintArgs* ca, const RkStage* rk) {
  b200bssn_ctx* ctx = P->ctx;
  DerivArgs da;
  AlgebraArgs aa;
  make_args(P, rhs, u, prm, da, aa);
  if (rk) aa.rk = *rk;
  if (P->single_pass && !ca) return launch_single_pass(P, da, aa, s, ev);
  const size_t nch = P->chunks.size();
  const bool pipelined = ev == nullptr && nch > 1;
  cudaStream_t s1 = pipelined ? ctx->s_deriv : s, s2 = pipelined ? ctx->s_alg : s;
  CK(ctx, cudaMemsetAsync(P->d_counters, 0, 2 * nch * sizeof(int), s));
  if (pipelined) {
    CK(ctx, cudaEventRecord(P->ev_fork, s));
    CK(ctx, cudaStreamWaitEvent(s1, P->ev_fork, 0));
    CK(ctx, cudaStreamWaitEvent(s2, P->ev_fork, 0));
  }
  for (size_t ci = 0; ci < nch; ++ci) {
    if (pipelined && ci >= 2) CK(ctx, cudaStreamWaitEvent(s1, P->ev_alg[ci - 2], 0));
    const int rc = enqueue_chunk(P, da, aa, ci, pipelined ? (int)(ci & 1) : 0, s1, s2, ev, ca);
    if (rc != B200BSSN_OK) return rc;
  }
  if (pipelined) CK(ctx, cudaStreamWaitEvent(s, P->ev_alg[nch - 1], 0));
  return B200BSSN_OK;
}

namespace {

int set_kernel_attributes(b200bssn_ctx* ctx) {
  int rc = set_stage_attributes<float, false>(ctx);
  if (rc == B200BSSN_OK) rc = set_stage_attributes<float, true>(ctx);
  if (rc == B200BSSN_OK) rc = set_stage_attributes<double, false>(ctx);
  if (rc == B200BSSN_OK) rc = set_stage_attributes<double, true>(ctx);
  if (rc != B200BSSN_OK) return rc;
  CK(ctx, cudaFuncSetAttribute(bssn_derivs_kernel<double>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDerivSmemBytes));
  CK(ctx, cudaFuncSetAttribute(bssn_derivs_kernel<float>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDerivSmemBytes));
  const int fb = (int)kFusedSmemBytes;
  CK(ctx, cudaFuncSetAttribute(bssn_fused_kernel<RK_NONE>, cudaFuncAttributeMaxDynamicSharedMemorySize, fb));
  CK(ctx, cudaFuncSetAttribute(bssn_fused_kernel<RK_FIRST>, cudaFuncAttributeMaxDynamicSharedMemorySize, fb));
  CK(ctx, cudaFuncSetAttribute(bssn_fused_kernel<RK_MIDDLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, fb));
  CK(ctx, cudaFuncSetAttribute(bssn_fused_kernel<RK_LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, fb));
  return B200BSSN_OK;
}

}  // namespace

extern "C" {

void b200bssn_default_params(b200bssn_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  for (int i = 0; i < 4; ++i) p->lambda[i] = 1;
  p->lambda_f[0] = 1.0;
  p->lambda_f[1] = 0.0;
  p->eta_const = 2.0;
  p->eta_r0 = 50.0;
  p->eta_damping_exp = 1.0;
  p->ko_sigma = 0.01;
  p->precision = B200BSSN_FP64;
  p->ghost_policy = B200BSSN_GHOSTS_PRESERVE;
}

const char* b200bssn_status_string(int s) {
  switch (s) {
    case B200BSSN_OK: return "ok";
    case B200BSSN_ERR_INVALID_ARGUMENT: return "invalid argument";
    case B200BSSN_ERR_BLOCK_TOO_SMALL: return "block interior below 7 points";
    case B200BSSN_ERR_CUDA: return "CUDA runtime error";
    case B200BSSN_ERR_OUT_OF_MEMORY: return "device out of memory";
    case B200BSSN_ERR_NO_DEVICE: return "no usable sm_100 device";
    case B200BSSN_ERR_NONFINITE: return "non-finite right-hand side";
    case B200BSSN_ERR_TIMEOUT: return "bounded device wait timed out";
    case B200BSSN_ERR_SIZE_LIMIT: return "request exceeds a fixed size limit";
    default: return "unknown status";
  }
}

int b200bssn_create(b200bssn_ctx** out, int device) {
  if (!out) return B200BSSN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return B200BSSN_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
    cudaGetLastError();
    return B200BSSN_ERR_NO_DEVICE;
  }
  b200bssn_ctx* ctx = new b200bssn_ctx();
  ctx->device = device;
  int rc = B200BSSN_OK;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->s_deriv, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->s_alg, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->s_h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->s_d2h, cudaStreamNonBlocking);
  if (e != cudaSuccess) rc = fail_cuda(ctx, e, "context setup");
  if (rc == B200BSSN_OK) rc = set_kernel_attributes(ctx);
  if (rc != B200BSSN_OK) {
    b200bssn_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return B200BSSN_OK;
}

int b200bssn_destroy(b200bssn_ctx* ctx) {
  if (!ctx) return B200BSSN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (ctx->blk_plan) b200bssn_plan_destroy(ctx->blk_plan);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->blk_u);
  cudaFree(ctx->blk_rhs);
  cudaFreeHost(ctx->blk_pin);
  for (cudaEvent_t e : ctx->blk_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->s_deriv) cudaStreamDestroy(ctx->s_deriv);
  if (ctx->s_alg) cudaStreamDestroy(ctx->s_alg);
  if (ctx->s_h2d) cudaStreamDestroy(ctx->s_h2d);
  if (ctx->s_d2h) cudaStreamDestroy(ctx->s_d2h);
  delete ctx;
  return B200BSSN_OK;
}

void* b200bssn_stream(b200bssn_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

const char* b200bssn_last_error(b200bssn_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int b200bssn_plan_create(b200bssn_ctx* ctx, const b200bssn_block* blocks, uint32_t nblocks,
                         uint32_t precision, uint64_t chunk_points, b200bssn_plan** out) {
  b200bssn_plan_options o;
  std::memset(&o, 0, sizeof(o));
  o.chunk_points = chunk_points;
  return b200bssn_plan_create_ex(ctx, blocks, nblocks, precision, &o, out);
}

int b200bssn_plan_create_ex(b200bssn_ctx* ctx, const b200bssn_block* blocks, uint32_t nblocks,
                            uint32_t precision, const b200bssn_plan_options* opts,
                            b200bssn_plan** out) {
  b200bssn_plan_options o;
  std::memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  const uint64_t chunk_points = o.chunk_points;
  const int64_t slab_depth = o.slab_depth ? (int64_t)o.slab_depth : kTileZ;
  if (!ctx || !blocks || !out || nblocks == 0) return B200BSSN_ERR_INVALID_ARGUMENT;
  if (precision != B200BSSN_FP64 && precision != B200BSSN_MIXED) return B200BSSN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  CK(ctx, cudaSetDevice(ctx->device));
  b200bssn_plan* P = new b200bssn_plan();
  P->ctx = ctx;
  P->precision = precision;
  P->advective = o.advective != 0;
  P->tile_y = o.tile_y ? (int)o.tile_y : kTileY;
  // register split: option 1 = 96/128 registers (the kinds without / with second
  // derivatives), 2 = 80/96, 3 = 128/168; 0 = the measured best for the precision
  // (FP64 with centred advection: 128/168, 4 % faster on the batch; else 96/128)
  const uint32_t regs_opt = o.deriv_regs ? o.deriv_regs
                                         : (precision == B200BSSN_FP64 && !P->advective && P->tile_y == kTileY ? 3u : 1u);
  P->deriv_regs = regs_opt >= 1 && regs_opt <= 3 ? (int)regs_opt - 1 : -1;  // kernel variant
  P->deriv_threads = kTileX * P->tile_y;
  for (int k = 0; k < 2; ++k)
    P->kind_fn[k] = kind_kernel(precision == B200BSSN_MIXED, P->advective, k == 1, P->tile_y, P->deriv_regs);
  if (o.points_per_thread == 2) {
    // y pairs: 16x16 tiles, 128 threads, centred advection, the pair kernels' own split
    const bool ok = !P->advective && (o.tile_y == 0 || o.tile_y == 16) && o.deriv_regs == 0;
    P->tile_y = 16;
    P->deriv_threads = 128;
    for (int k = 0; k < 2; ++k)
      P->kind_fn[k] = !ok ? nullptr
                          : (precision == B200BSSN_MIXED
                                 ? (k ? (const void*)bssn_derivs_pair_kernel<float, true>
                                      : (const void*)bssn_derivs_pair_kernel<float, false>)
                                 : (k ? (const void*)bssn_derivs_pair_kernel<double, true>
                                      : (const void*)bssn_derivs_pair_kernel<double, false>));
  } else if (o.points_per_thread > 2) {
    P->kind_fn[0] = P->kind_fn[1] = nullptr;
  }
  if (!P->kind_fn[0] || !P->kind_fn[1]) {
    delete P;
    return B200BSSN_ERR_INVALID_ARGUMENT;
  }
  const int nslots = P->advective ? kNumDerivs + 3 * kNumVars : kNumDerivs;
  const int64_t kMaxChunkPoints = max_chunk_points(nslots);
  P->span_lo = UINT64_MAX;
  int64_t max_unit = 0;
  for (uint32_t b = 0; b < nblocks; ++b) {
    const b200bssn_block& in = blocks[b];
    for (int a = 0; a < 3; ++a) {
      if (in.sz[a] < 13) {
        delete P;
        return B200BSSN_ERR_BLOCK_TOO_SMALL;
      }
      if (in.sz[a] > 32767 || !(in.pmax[a] > in.pmin[a])) {
        delete P;
        return B200BSSN_ERR_INVALID_ARGUMENT;
      }
    }
    if (in.bflag >> 6) {
      delete P;
      return B200BSSN_ERR_INVALID_ARGUMENT;
    }
    BlockDev d;
    d.offset = in.offset;
    d.bflag = in.bflag;
    for (int a = 0; a < 3; ++a) {
      d.sz[a] = (int32_t)in.sz[a];
      d.pmin[a] = in.pmin[a];
      d.h[a] = (in.pmax[a] - in.pmin[a]) / (in.sz[a] - 1);  // rhs.cpp:144-146
    }
    P->blocks.push_back(d);
    const uint64_t npad = (uint64_t)in.sz[0] * in.sz[1] * in.sz[2];
    P->span_lo = std::min<uint64_t>(P->span_lo, in.offset);
    P->span_hi = std::max<uint64_t>(P->span_hi, in.offset + npad);
    const int64_t I0 = in.sz[0] - 6, I1 = in.sz[1] - 6, I2 = in.sz[2] - 6;
    // z-slabs of nearly equal depth (<= depth planes): the derivative kernel
    // streams each slab plus 4 halo planes on each side
    const int64_t depth = (o.block_slab_depth && o.block_slab_depth[b])
                              ? (int64_t)o.block_slab_depth[b] : slab_depth;
    const int64_t nslab = (I2 + depth - 1) / depth;
    if ((uint64_t)I0 * I1 * ((I2 + nslab - 1) / nslab) > (uint64_t)INT32_MAX) {
      delete P;
      return B200BSSN_ERR_INVALID_ARGUMENT;
    }
    for (int64_t sl = 0; sl < nslab; ++sl) {
      const int64_t k0 = sl * I2 / nslab, k1 = (sl + 1) * I2 / nslab;
      UnitDev u;
      u.block = (int32_t)b;
      u.k0 = (int32_t)k0;
      u.nz = (int32_t)(k1 - k0);
      u.pad = 0;
      u.sbase = 0;
      P->units.push_back(u);
      max_unit = std::max<int64_t>(max_unit, I0 * I1 * u.nz);
    }
    P->points += (uint64_t)(I0 * I1 * I2);
  }
  int64_t capacity = chunk_points ? (int64_t)chunk_points : kDefaultChunkPoints;
  capacity = std::min(std::max(capacity, max_unit), kMaxChunkPoints);
  if (max_unit > kMaxChunkPoints) {
    delete P;
    return B200BSSN_ERR_SIZE_LIMIT;
  }
  // pack units into chunks
  ChunkRec cur{0, 0, 0, 0, 0};
  auto flush = [&]() {
    if (cur.points > 0) {
      cur.tile_count = (int32_t)P->tiles.size() - cur.tile_begin;
      cur.range_count = (int32_t)P->ranges.size() - cur.range_begin;
      P->chunks.push_back(cur);
      P->cap = std::max<int64_t>(P->cap, (cur.points + 31) & ~int64_t(31));
    }
    cur = ChunkRec{(int32_t)P->tiles.size(), 0, (int32_t)P->ranges.size(), 0, 0};
  };
  for (size_t ui = 0; ui < P->units.size(); ++ui) {
    UnitDev& u = P->units[ui];
    const BlockDev& B = P->blocks[u.block];
    const int I0 = B.sz[0] - 6, I1 = B.sz[1] - 6;
    const int64_t np = (int64_t)I0 * I1 * u.nz;
    // a block's units stay in one chunk when the whole block fits in one
    const int64_t block_pts = (int64_t)I0 * I1 * (B.sz[2] - 6);
    const bool first_unit = ui == 0 || P->units[ui - 1].block != u.block;
    if (first_unit && block_pts <= capacity && cur.points + block_pts > capacity) flush();
    if (((cur.points + 31) & ~int64_t(31)) + np > capacity) flush();
    cur.points = (cur.points + 31) & ~int64_t(31);  // slot runs start 128-byte aligned
    u.sbase = cur.points;
    cur.points += np;
    for (int j0 = 0; j0 < I1; j0 += P->tile_y)
      for (int i0 = 0; i0 < I0; i0 += kTileX) {
        TileDev t;
        t.unit = (int32_t)ui;
        t.i0 = (int16_t)i0;
        t.j0 = (int16_t)j0;
        t.ex = (int16_t)std::min(kTileX, I0 - i0);
        t.ey = (int16_t)std::min(P->tile_y, I1 - j0);
        P->tiles.push_back(t);
      }
    for (int64_t s = 0; s < np; s += kAlgebraThreads) {
      RangeDev r;
      r.unit = (int32_t)ui;
      r.start = (int32_t)s;
      r.count = (int32_t)std::min<int64_t>(kAlgebraThreads, np - s);
      P->ranges.push_back(r);
    }
  }
  flush();
  // Host pipeline partition: chunk c owns elements [part[c], part[c+1]) when the
  // chunks' blocks are disjoint and in increasing offset order.
  {
    std::vector<uint64_t> lo(P->chunks.size(), UINT64_MAX), hi(P->chunks.size(), 0);
    P->chunk_blocks.assign(P->chunks.size(), {});
    for (size_t c = 0; c < P->chunks.size(); ++c) {
      const ChunkRec& ch = P->chunks[c];
      for (int r = ch.range_begin; r < ch.range_begin + ch.range_count; ++r) {
        const int32_t bi = P->units[P->ranges[r].unit].block;
        const BlockDev& B = P->blocks[bi];
        const uint64_t np = (uint64_t)B.sz[0] * B.sz[1] * B.sz[2];
        lo[c] = std::min(lo[c], B.offset);
        hi[c] = std::max(hi[c], B.offset + np);
        if (P->chunk_blocks[c].empty() || P->chunk_blocks[c].back() != bi) P->chunk_blocks[c].push_back(bi);
      }
    }
    bool ok = P->chunks.size() > 1;
    for (size_t c = 0; ok && c + 1 < P->chunks.size(); ++c) ok = hi[c] <= lo[c + 1];
    if (ok) {
      P->part.resize(P->chunks.size() + 1);
      P->part[0] = P->span_lo;
      for (size_t c = 1; c < P->chunks.size(); ++c) P->part[c] = lo[c];
      P->part[P->chunks.size()] = P->span_hi;
      P->host_pipeline = true;
    }
  }
  // longest tiles first within each chunk (cost ~ planes streamed)
  for (const ChunkRec& c : P->chunks) {
    auto planes = [&](const TileDev& t) {
      const UnitDev& u = P->units[t.unit];
      const BlockDev& B = P->blocks[u.block];
      return std::min(B.sz[2], 3 + u.k0 + u.nz + kHalo) - std::max(0, 3 + u.k0 - kHalo);
    };
    std::stable_sort(P->tiles.begin() + c.tile_begin, P->tiles.begin() + c.tile_begin + c.tile_count,
                     [&](const TileDev& x, const TileDev& y) { return planes(x) > planes(y); });
  }
  {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const bool mx = precision == B200BSSN_MIXED, adv = P->advective;
    for (int k = 0; k < 2; ++k) {
      int per_sm = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, P->kind_fn[k], P->deriv_threads, 0);
      if (o.deriv_ctas_per_sm) per_sm = std::min<int>(per_sm, (int)o.deriv_ctas_per_sm);
      P->deriv_grid[k] = std::max(1, sms * std::max(1, per_sm));
    }
    int alg_per_sm = 0;
    if (mx && !adv)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&alg_per_sm, bssn_algebra_staged_kernel<float, RK_NONE, false>,
                                                    StageCfg<float, false>::kThreads, StageCfg<float, false>::kSmemBytes);
    else if (mx)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&alg_per_sm, bssn_algebra_staged_kernel<float, RK_NONE, true>,
                                                    StageCfg<float, true>::kThreads, StageCfg<float, true>::kSmemBytes);
    else if (!adv)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&alg_per_sm, bssn_algebra_staged_kernel<double, RK_NONE, false>,
                                                    StageCfg<double, false>::kThreads, StageCfg<double, false>::kSmemBytes);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&alg_per_sm, bssn_algebra_staged_kernel<double, RK_NONE, true>,
                                                    StageCfg<double, true>::kThreads, StageCfg<double, true>::kSmemBytes);
    P->alg_grid = std::max(1, sms * std::max(1, alg_per_sm));
  }

  // one-pass path (when asked for): MIXED with centred advection.  Tile-slabs of the
  // largest blocks first (the launch ends on small items); within a block, slab by
  // slab and tile by tile, so neighbouring items share halos.
  P->single_pass = precision == B200BSSN_MIXED && !P->advective && o.single_pass;
  if (P->single_pass) {
    P->nring = o.ring_slots ? (int32_t)std::min<uint32_t>(o.ring_slots, 1024) : kFusedRingDefault;
    std::vector<uint32_t> order(nblocks);
    for (uint32_t b = 0; b < nblocks; ++b) order[b] = b;
    auto npad = [&](uint32_t b) {
      const BlockDev& B = P->blocks[b];
      return (int64_t)B.sz[0] * B.sz[1] * B.sz[2];
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return npad(x) > npad(y); });
    int64_t groups = 0;  // planes over all tile-slabs (algebra work units)
    for (uint32_t b : order) {
      const BlockDev& B = P->blocks[b];
      const int I0 = B.sz[0] - 6, I1 = B.sz[1] - 6, I2 = B.sz[2] - 6;
      const int nslab = (I2 + kFusedSlab - 1) / kFusedSlab;
      for (int sl = 0; sl < nslab; ++sl) {
        const int k0 = (int)((int64_t)sl * I2 / nslab), k1 = (int)((int64_t)(sl + 1) * I2 / nslab);
        for (int j0 = 0; j0 < I1; j0 += kTileY)
          for (int i0 = 0; i0 < I0; i0 += kTileX) {
            FusedTileDev t;
            t.block = (int32_t)b;
            t.i0 = (int16_t)i0;
            t.j0 = (int16_t)j0;
            t.ex = (int16_t)std::min(kTileX, I0 - i0);
            t.ey = (int16_t)std::min(kTileY, I1 - j0);
            t.k0 = (int16_t)k0;
            t.nz = (int16_t)(k1 - k0);
            t.pad = 0;
            groups += t.nz;
            P->ftiles.push_back(t);
          }
      }
    }
    if (groups >= INT32_MAX || (int64_t)P->ftiles.size() * kNumVars >= INT32_MAX) {
      delete P;
      return B200BSSN_ERR_SIZE_LIMIT;
    }
    P->fsync_words = 4 + 3 * P->ftiles.size() + (size_t)P->nring;
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bssn_fused_kernel<RK_NONE>, kFusedThreads,
                                                  kFusedSmemBytes);
    P->fused_grid = std::max(1, sms * std::max(1, per_sm));
  }

  const size_t nb = P->blocks.size() * sizeof(BlockDev), nu = P->units.size() * sizeof(UnitDev),
               nt = P->tiles.size() * sizeof(TileDev), nr = P->ranges.size() * sizeof(RangeDev);
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t total = al(nb) + al(nu) + al(nt) + al(nr);
  cudaError_t e = cudaMalloc(&P->desc, total);
  const size_t st = precision == B200BSSN_MIXED ? sizeof(float) : sizeof(double);
  const int nbuf = P->chunks.size() > 1 ? 2 : 1;
  for (int b = 0; b < nbuf && e == cudaSuccess; ++b) {
    // + 512 B: the algebra kernels' copies and prefetches of a slot run are whole
    // 16-byte chunks or 32-point columns and may read past the last run's end
    e = cudaMalloc(&P->dscr[b], (size_t)nslots * P->cap * st + 512);
    if (e == cudaSuccess) e = cudaMalloc(&P->koscr[b], (size_t)kNumVars * P->cap * st + 512);
  }
  if (e == cudaSuccess && P->single_pass) {
    const size_t ntb = al(P->ftiles.size() * sizeof(FusedTileDev));
    e = cudaMalloc(&P->fdesc, ntb + al(P->fsync_words * sizeof(int)));
    if (e == cudaSuccess) {
      char* fb = static_cast<char*>(P->fdesc);
      P->d_ftiles = reinterpret_cast<FusedTileDev*>(fb);
      P->d_fsync = reinterpret_cast<int*>(fb + ntb);
      e = cudaMemcpy(P->d_ftiles, P->ftiles.data(), P->ftiles.size() * sizeof(FusedTileDev),
                     cudaMemcpyHostToDevice);
    }
    const size_t ring_pts = (size_t)P->nring * kFusedSlotPts;
    if (e == cudaSuccess) e = cudaMalloc(&P->fring_d, ring_pts * kNumDerivs * sizeof(float) + 512);
    if (e == cudaSuccess) e = cudaMalloc(&P->fring_k, ring_pts * kNumVars * sizeof(float) + 512);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc((void**)&P->d_counters, 2 * P->chunks.size() * sizeof(int));
  P->ev_deriv.assign(P->chunks.size(), nullptr);
  P->ev_alg.assign(P->chunks.size(), nullptr);
  P->ev_in.assign(P->chunks.size(), nullptr);
  for (size_t c = 0; c < P->chunks.size() && e == cudaSuccess; ++c) {
    e = cudaEventCreateWithFlags(&P->ev_deriv[c], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->ev_alg[c], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->ev_in[c], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    int rc = fail_cuda(ctx, e, "plan allocation");
    b200bssn_plan_destroy(P);
    return rc;
  }
  char* base = static_cast<char*>(P->desc);
  P->d_blocks = reinterpret_cast<BlockDev*>(base);
  P->d_units = reinterpret_cast<UnitDev*>(base + al(nb));
  P->d_tiles = reinterpret_cast<TileDev*>(base + al(nb) + al(nu));
  P->d_ranges = reinterpret_cast<RangeDev*>(base + al(nb) + al(nu) + al(nt));
  e = cudaMemcpy(P->d_blocks, P->blocks.data(), nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(P->d_units, P->units.data(), nu, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(P->d_tiles, P->tiles.data(), nt, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(P->d_ranges, P->ranges.data(), nr, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    int rc = fail_cuda(ctx, e, "plan upload");
    b200bssn_plan_destroy(P);
    return rc;
  }
  *out = P;
  return B200BSSN_OK;
}

int b200bssn_plan_destroy(b200bssn_plan* P) {
  if (!P) return B200BSSN_ERR_INVALID_ARGUMENT;
  if (P->ctx) cudaSetDevice(P->ctx->device);
  cudaFree(P->desc);
  if (P->ctx && P->ctx->stream) {
    cudaStreamSynchronize(P->ctx->s_deriv);
    cudaStreamSynchronize(P->ctx->s_alg);
    cudaStreamSynchronize(P->ctx->s_h2d);
    cudaStreamSynchronize(P->ctx->s_d2h);
  }
  for (int b = 0; b < 2; ++b) {
    cudaFree(P->dscr[b]);
    cudaFree(P->koscr[b]);
  }
  for (cudaEvent_t e : P->ev_deriv)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : P->ev_alg)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : P->ev_in)
    if (e) cudaEventDestroy(e);
  if (P->ev_fork) cudaEventDestroy(P->ev_fork);
  cudaFree(P->d_counters);
  cudaFree(P->d_guard);
  cudaFree(P->fdesc);
  cudaFree(P->fring_d);
  cudaFree(P->fring_k);
  cudaFree(P->st_u);
  cudaFree(P->st_rhs);
  delete P;
  return B200BSSN_OK;
}

uint64_t b200bssn_plan_points(const b200bssn_plan* P) { return P ? P->points : 0; }

uint32_t b200bssn_plan_launches(const b200bssn_plan* P) {
  if (!P) return 0;
  if (P->single_pass) return 1;                 // the one-pass kernel
  return (uint32_t)(3 * P->chunks.size());      // two derivative kernels + algebra per chunk
}

uint32_t b200bssn_plan_single_pass(const b200bssn_plan* P) { return P && P->single_pass ? 1u : 0u; }

int b200bssn_plan_status(b200bssn_plan* P) {
  if (!P) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = P->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  CK(ctx, cudaDeviceSynchronize());
  if (!P->single_pass) return B200BSSN_OK;
  int err = 0;
  CK(ctx, cudaMemcpy(&err, P->d_fsync + 2, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    ctx->last_error = "one-pass kernel: a bounded wait for work timed out";
    return B200BSSN_ERR_TIMEOUT;
  }
  return B200BSSN_OK;
}

int b200bssn_rhs_plan_device(b200bssn_plan* P, double* const* rhs_dev, const double* const* u_dev,
                             const b200bssn_params* prm, void* stream) {
  b200bssn::host::NvtxRange nvtx_("b200bssn_rhs_plan_device");
  if (!P || !rhs_dev || !u_dev || !params_ok(prm)) return B200BSSN_ERR_INVALID_ARGUMENT;
  if (prm->precision != P->precision) return B200BSSN_ERR_INVALID_ARGUMENT;
  for (int v = 0; v < kNumVars; ++v)
    if (!rhs_dev[v] || !u_dev[v]) return B200BSSN_ERR_INVALID_ARGUMENT;
  cudaStream_t s = stream ? (cudaStream_t)stream : P->ctx->stream;
  return launch_plan(P, rhs_dev, u_dev, prm, s);
}

int b200bssn_plan_profile(b200bssn_plan* P, double* const* rhs_dev, const double* const* u_dev,
                          const b200bssn_params* prm, double* ms_deriv, double* ms_algebra) {
  if (!P || !rhs_dev || !u_dev || !params_ok(prm) || !ms_deriv || !ms_algebra)
    return B200BSSN_ERR_INVALID_ARGUMENT;
  if (prm->precision != P->precision) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = P->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  if (P->single_pass) {
    // one kernel: its whole time is reported as the derivative part, 0 as the algebra
    cudaEvent_t ev[2];
    CK(ctx, cudaEventCreate(&ev[0]));
    CK(ctx, cudaEventCreate(&ev[1]));
    int rc = launch_plan(P, rhs_dev, u_dev, prm, ctx->stream, ev);
    float t = 0;
    if (rc == B200BSSN_OK) {
      cudaError_t e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) rc = fail_cuda(ctx, e, "profile sync");
      else cudaEventElapsedTime(&t, ev[0], ev[1]);
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    *ms_deriv = t;
    *ms_algebra = 0.0;
    return rc;
  }
  std::vector<cudaEvent_t> ev(4 * P->chunks.size());
  for (auto& e : ev) CK(ctx, cudaEventCreate(&e));
  int rc = launch_plan(P, rhs_dev, u_dev, prm, ctx->stream, ev.data());
  if (rc == B200BSSN_OK) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = fail_cuda(ctx, e, "profile sync");
  }
  double d = 0, a = 0;
  for (size_t c = 0; rc == B200BSSN_OK && c < P->chunks.size(); ++c) {
    float t1 = 0, t2 = 0;
    cudaEventElapsedTime(&t1, ev[4 * c + 0], ev[4 * c + 1]);
    cudaEventElapsedTime(&t2, ev[4 * c + 2], ev[4 * c + 3]);
    d += t1;
    a += t2;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  *ms_deriv = d;
  *ms_algebra = a;
  return rc;
}

}  // extern "C"

namespace {

// Pipelined host path: per chunk c, the upload of its element range (stream
// s_h2d), its two kernels (s_deriv, s_alg) and the download of its range of the
// RHS (s_d2h), with event edges upload(c) -> K1(c) -> K2(c) -> download(c) and
// K2(c-2) -> K1(c) (scratch reuse).  Uploads, kernels and downloads of different
// chunks overlap; both copy directions run at once.
// Interior x-extent (points) from which a block's result comes back as a strided box
// copy on the ghost-preserving host path (37^3 blocks and up; 13^3 and 21^3 blocks,
// with rows of 7 and 15 points, come back whole with their ghosts uploaded first).
constexpr int kBoxCopyMinRow = 24;

// Enqueues the copy of block B's interior box [3, n-3)^3 from the device array `src`
// to the host array `dst` (both indexed by the caller's element numbering).
cudaError_t copy_box_d2h(double* dst, const double* src, const BlockDev& B, cudaStream_t s) {
  const size_t nx = B.sz[0], ny = B.sz[1];
  cudaMemcpy3DParms cp;
  std::memset(&cp, 0, sizeof(cp));
  cp.srcPtr = make_cudaPitchedPtr(const_cast<double*>(src) + B.offset, nx * sizeof(double), nx, ny);
  cp.dstPtr = make_cudaPitchedPtr(dst + B.offset, nx * sizeof(double), nx, ny);
  cp.srcPos = make_cudaPos(3 * sizeof(double), 3, 3);
  cp.dstPos = cp.srcPos;
  cp.extent = make_cudaExtent((nx - 6) * sizeof(double), ny - 6, B.sz[2] - 6);
  cp.kind = cudaMemcpyDeviceToHost;
  return cudaMemcpy3DAsync(&cp, s);
}

int host_pipelined(b200bssn_plan* P, double* const* rhs, const double* const* u, double* const* rd,
                   const double* const* ud, const b200bssn_params* prm) {
  b200bssn_ctx* ctx = P->ctx;
  DerivArgs da;
  AlgebraArgs aa;
  make_args(P, rd, ud, prm, da, aa);
  const size_t nch = P->chunks.size();
  const bool preserve = prm->ghost_policy == B200BSSN_GHOSTS_PRESERVE;
  cudaStream_t sin = ctx->s_h2d, s1 = ctx->s_deriv, s2 = ctx->s_alg, sout = ctx->s_d2h;
  CK(ctx, cudaMemsetAsync(P->d_counters, 0, 2 * nch * sizeof(int), s1));
  for (size_t ci = 0; ci < nch; ++ci) {
    const uint64_t a = P->part[ci], b = P->part[ci + 1];
    const size_t nb = (size_t)(b - a) * sizeof(double);
    // PRESERVE: the interior boxes of large blocks come back by strided copies into the
    // caller's arrays, so their ghost values are never touched; runs of consecutive small
    // blocks (rows too short for strided copies to pay) go up with the caller's RHS values
    // and come back whole, so their ghosts return unchanged
    std::vector<int32_t> boxes;
    std::vector<std::pair<uint64_t, uint64_t>> runs;
    if (preserve) {
      for (const int32_t bi : P->chunk_blocks[ci]) {
        const BlockDev& B = P->blocks[bi];
        const uint64_t lo = B.offset, hi = B.offset + (uint64_t)B.sz[0] * B.sz[1] * B.sz[2];
        if (B.sz[0] - 6 >= kBoxCopyMinRow)
          boxes.push_back(bi);
        else if (!runs.empty() && runs.back().second <= lo && lo - runs.back().second < 64)
          runs.back().second = hi;  // the gap is alignment padding of the caller's arrays
        else
          runs.emplace_back(lo, hi);
      }
    }
    for (int v = 0; v < kNumVars; ++v) {
      // (ZERO: st_rhs was cleared once, before the first chunk; the kernels write
      // interior points only)
      CK(ctx, cudaMemcpyAsync((void*)(ud[v] + a), u[v] + a, nb, cudaMemcpyHostToDevice, sin));
      for (const auto& r : runs)
        CK(ctx, cudaMemcpyAsync(rd[v] + r.first, rhs[v] + r.first, (r.second - r.first) * sizeof(double),
                                cudaMemcpyHostToDevice, sin));
    }
    CK(ctx, cudaEventRecord(P->ev_in[ci], sin));
    CK(ctx, cudaStreamWaitEvent(s1, P->ev_in[ci], 0));
    if (ci >= 2) CK(ctx, cudaStreamWaitEvent(s1, P->ev_alg[ci - 2], 0));
    const int rc = enqueue_chunk(P, da, aa, ci, (int)(ci & 1), s1, s2, nullptr);
    if (rc != B200BSSN_OK) return rc;
    CK(ctx, cudaStreamWaitEvent(sout, P->ev_alg[ci], 0));
    if (preserve) {
      for (const int32_t bi : boxes)
        for (int v = 0; v < kNumVars; ++v) CK(ctx, copy_box_d2h(rhs[v], rd[v], P->blocks[bi], sout));
      for (const auto& r : runs)
        for (int v = 0; v < kNumVars; ++v)
          CK(ctx, cudaMemcpyAsync(rhs[v] + r.first, rd[v] + r.first, (r.second - r.first) * sizeof(double),
                                  cudaMemcpyDeviceToHost, sout));
    } else {
      for (int v = 0; v < kNumVars; ++v)
        CK(ctx, cudaMemcpyAsync(rhs[v] + a, rd[v] + a, nb, cudaMemcpyDeviceToHost, sout));
    }
  }
  CK(ctx, cudaStreamSynchronize(sout));
  CK(ctx, cudaStreamSynchronize(s1));
  CK(ctx, cudaStreamSynchronize(sin));
  return B200BSSN_OK;
}

}  // namespace

extern "C" {

int b200bssn_rhs_plan_host(b200bssn_plan* P, double* const* rhs, const double* const* u,
                           uint64_t n_elems, const b200bssn_params* prm) {
  b200bssn::host::NvtxRange nvtx_("b200bssn_rhs_plan_host");
  if (!P || !rhs || !u || !params_ok(prm)) return B200BSSN_ERR_INVALID_ARGUMENT;
  if (prm->precision != P->precision || n_elems < P->span_hi) return B200BSSN_ERR_INVALID_ARGUMENT;
  for (int v = 0; v < kNumVars; ++v)
    if (!rhs[v] || !u[v]) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = P->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  const uint64_t len = P->span_hi - P->span_lo;
  if (P->st_len < len) {
    cudaFree(P->st_u);
    cudaFree(P->st_rhs);
    P->st_u = P->st_rhs = nullptr;
    P->st_len = 0;
    CK(ctx, cudaMalloc((void**)&P->st_u, (size_t)kNumVars * len * sizeof(double)));
    CK(ctx, cudaMalloc((void**)&P->st_rhs, (size_t)kNumVars * len * sizeof(double)));
    P->st_len = len;
    P->st_rhs_zeroed = false;
  }
  cudaStream_t s = ctx->stream;
  const double* ud[kNumVars];
  double* rd[kNumVars];
  const size_t bytes = len * sizeof(double);
  for (int v = 0; v < kNumVars; ++v) {
    // device arrays are shifted so that element `span_lo` lands at the start
    ud[v] = P->st_u + (size_t)v * len - P->span_lo;
    rd[v] = P->st_rhs + (size_t)v * len - P->span_lo;
  }
  if (prm->ghost_policy == B200BSSN_GHOSTS_PRESERVE) {
    P->st_rhs_zeroed = false;  // the caller's RHS values go into st_rhs below
  } else if (!P->st_rhs_zeroed) {
    CK(ctx, cudaMemsetAsync(P->st_rhs, 0, (size_t)kNumVars * bytes, P->host_pipeline ? ctx->s_h2d : s));
    P->st_rhs_zeroed = true;
  }
  if (P->host_pipeline) return host_pipelined(P, rhs, u, rd, ud, prm);
  for (int v = 0; v < kNumVars; ++v) {
    CK(ctx, cudaMemcpyAsync(P->st_u + (size_t)v * len, u[v] + P->span_lo, bytes,
                            cudaMemcpyHostToDevice, s));
    if (prm->ghost_policy == B200BSSN_GHOSTS_PRESERVE)
      CK(ctx, cudaMemcpyAsync(P->st_rhs + (size_t)v * len, rhs[v] + P->span_lo, bytes,
                              cudaMemcpyHostToDevice, s));
  }
  int rc = launch_plan(P, rd, ud, prm, s);
  if (rc != B200BSSN_OK) return rc;
  for (int v = 0; v < kNumVars; ++v)
    CK(ctx, cudaMemcpyAsync(rhs[v] + P->span_lo, P->st_rhs + (size_t)v * len, bytes,
                            cudaMemcpyDeviceToHost, s));
  CK(ctx, cudaStreamSynchronize(s));
  return B200BSSN_OK;
}

}  // extern "C"

namespace {

// Drop-in calls in flight in this process: a host code may call the drop-in from
// many threads at once (each with its own context, as the reference's OpenMP block
// loop calls bssnrhs), and they share the host's cores for their staging copies.
std::atomic<int> g_dropin_calls{0};
struct DropinCall {
  DropinCall() { g_dropin_calls.fetch_add(1); }
  ~DropinCall() { g_dropin_calls.fetch_sub(1); }
  DropinCall(const DropinCall&) = delete;
  DropinCall& operator=(const DropinCall&) = delete;
};

// Blocks whose 24 variables take at most this many bytes go up in one copy and come
// back in one (the per-copy cost outweighs the ghost planes copied along).
constexpr size_t kSmallBlockBytes = size_t(8) << 20;

// Host threads for staging `bytes` of block data: one per 4 MB, at most 8 and at
// most this call's share of the host's hardware threads.
int staging_threads(size_t bytes) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned share = std::max(1u, hw / (unsigned)std::max(1, g_dropin_calls.load()));
  return (int)std::min<size_t>({8, share, bytes / (4u << 20) + 1});
}

// Runs fn(i) for i in [0, n) on up to `threads` host threads (the calling thread
// among them; each worker selects `device` first) and returns the first CUDA error.
// Workers that cannot be started leave their share to the others.
template <class F>
cudaError_t host_parallel(int device, int n, int threads, F fn) {
  std::atomic<int> next{0};
  std::atomic<int> err{(int)cudaSuccess};
  auto work = [&](bool worker) {
    if (worker) {
      const cudaError_t e = cudaSetDevice(device);
      if (e != cudaSuccess) {
        int ok = (int)cudaSuccess;
        err.compare_exchange_strong(ok, (int)e);
        return;
      }
    }
    for (int i; (i = next.fetch_add(1)) < n;) {
      const cudaError_t e = fn(i);
      if (e != cudaSuccess) {
        int ok = (int)cudaSuccess;
        err.compare_exchange_strong(ok, (int)e);
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < std::min(threads, n); ++t) {
    try {
      pool.emplace_back(work, true);
    } catch (const std::system_error&) {
      break;
    }
  }
  work(false);
  for (std::thread& t : pool) t.join();
  return (cudaError_t)err.load();
}

// Single-block path shared by the drop-in entry points: (re)builds the one-block
// plan when the size or precision changes (otherwise only the block descriptor is
// refreshed), sizes the block buffers and uploads the block's state.  On return
// ud/rd point at the device copies of u and at a [24][npad] output buffer.
int prepare_block(b200bssn_ctx* ctx, const double* const* u, uint32_t offset, const double* pmin,
                  const double* pmax, const uint32_t* sz, uint32_t bflag, uint32_t precision,
                  const double** ud, double** rd) {
  CK(ctx, cudaSetDevice(ctx->device));
  // the pinned buffer is free once the context's earlier copies are done (a call
  // that returned an error may have left some in flight)
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  b200bssn_block blk;
  blk.offset = 0;
  blk.bflag = bflag;
  for (int a = 0; a < 3; ++a) {
    blk.sz[a] = sz[a];
    blk.pmin[a] = pmin[a];
    blk.pmax[a] = pmax[a];
  }
  const size_t npad = (size_t)sz[0] * sz[1] * sz[2];
  if (!ctx->blk_plan || std::memcmp(ctx->blk_sz, sz, sizeof(ctx->blk_sz)) != 0 ||
      ctx->blk_precision != precision) {
    if (ctx->blk_plan) b200bssn_plan_destroy(ctx->blk_plan);
    ctx->blk_plan = nullptr;
    int rc = b200bssn_plan_create(ctx, &blk, 1, precision, 0, &ctx->blk_plan);
    if (rc != B200BSSN_OK) return rc;
    std::memcpy(ctx->blk_sz, sz, sizeof(ctx->blk_sz));
    ctx->blk_precision = precision;
  } else {
    if (bflag >> 6) return B200BSSN_ERR_INVALID_ARGUMENT;
    for (int a = 0; a < 3; ++a)
      if (!(pmax[a] > pmin[a])) return B200BSSN_ERR_INVALID_ARGUMENT;
    BlockDev& d = ctx->blk_plan->blocks[0];
    d.bflag = bflag;
    for (int a = 0; a < 3; ++a) {
      d.pmin[a] = pmin[a];
      d.h[a] = (pmax[a] - pmin[a]) / (sz[a] - 1);
    }
    CK(ctx, cudaMemcpyAsync(ctx->blk_plan->d_blocks, &d, sizeof(BlockDev), cudaMemcpyHostToDevice,
                            ctx->stream));
  }
  if (ctx->blk_cap < npad) {
    cudaFree(ctx->blk_u);
    cudaFree(ctx->blk_rhs);
    ctx->blk_u = ctx->blk_rhs = nullptr;
    ctx->blk_cap = 0;
    CK(ctx, cudaMalloc((void**)&ctx->blk_u, kNumVars * npad * sizeof(double)));
    CK(ctx, cudaMalloc((void**)&ctx->blk_rhs, kNumVars * npad * sizeof(double)));
    ctx->blk_cap = npad;
  }
  if (ctx->blk_pin_cap < kNumVars * npad) {
    CK(ctx, cudaFreeHost(ctx->blk_pin));
    ctx->blk_pin = nullptr;
    ctx->blk_pin_cap = 0;
    CK(ctx, cudaHostAlloc((void**)&ctx->blk_pin, kNumVars * npad * sizeof(double),
                          cudaHostAllocDefault));
    ctx->blk_pin_cap = kNumVars * npad;
  }
  for (int v = 0; v < kNumVars; ++v) {
    ud[v] = ctx->blk_u + v * npad;
    rd[v] = ctx->blk_rhs + v * npad;
  }
  double* pin = ctx->blk_pin;
  double* dev = ctx->blk_u;
  cudaStream_t s = ctx->stream;
  const size_t bytes = npad * sizeof(double);
  if (kNumVars * bytes <= kSmallBlockBytes) {
    // small block: one host copy per variable into the pinned buffer, one upload
    for (int v = 0; v < kNumVars; ++v) std::memcpy(pin + v * npad, u[v] + offset, bytes);
    CK(ctx, cudaMemcpyAsync(dev, pin, kNumVars * bytes, cudaMemcpyHostToDevice, s));
    return B200BSSN_OK;
  }
  // each variable goes through the pinned buffer; its upload is queued as soon as
  // its host copy is done, so the DMA of one variable overlaps the copy of the next
  const cudaError_t e = host_parallel(
      ctx->device, kNumVars, staging_threads(kNumVars * bytes), [=](int v) {
        std::memcpy(pin + v * npad, u[v] + offset, bytes);
        return cudaMemcpyAsync(dev + v * npad, pin + v * npad, bytes, cudaMemcpyHostToDevice, s);
      });
  if (e != cudaSuccess) return fail_cuda(ctx, e, "block upload");
  return B200BSSN_OK;
}

// Copies the interior box [3, n-3)^3 of `nout` device arrays back to the caller's
// host arrays at `offset`; ghost points of the destination are left untouched, as
// the reference leaves them.  Each variable's interior planes come down as one
// contiguous copy into the pinned buffer, and host threads scatter its interior rows
// as soon as its copy is done.
int copy_interior_back(b200bssn_ctx* ctx, double* const* dst, double* const* src, int nout,
                       uint32_t offset, const uint32_t* sz) {
  const size_t nx = sz[0], ny = sz[1], nz = sz[2];
  const size_t plane = nx * ny, npad = plane * nz;
  const size_t lo = 3 * plane, n = (nz - 6) * plane;
  const size_t row = (nx - 6) * sizeof(double);
  auto scatter = [&](int v) {
    const double* from = ctx->blk_pin + v * npad;
    double* to = dst[v] + offset;
    for (size_t k = 3; k < nz - 3; ++k)
      for (size_t j = 3; j < ny - 3; ++j) {
        const size_t at = k * plane + j * nx + 3;
        std::memcpy(to + at, from + at, row);
      }
  };
  bool contiguous = true;  // the outputs are consecutive arrays of the block buffer
  for (int v = 1; v < nout; ++v) contiguous = contiguous && src[v] == src[0] + v * npad;
  if (contiguous && nout * npad * sizeof(double) <= kSmallBlockBytes) {
    // small block: one download of the whole output, then the row scatter
    CK(ctx, cudaMemcpyAsync(ctx->blk_pin, src[0], nout * npad * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    for (int v = 0; v < nout; ++v) scatter(v);
    return B200BSSN_OK;
  }
  for (int v = 0; v < nout; ++v) {
    if (!ctx->blk_ev[v]) CK(ctx, cudaEventCreateWithFlags(&ctx->blk_ev[v], cudaEventDisableTiming));
    CK(ctx, cudaMemcpyAsync(ctx->blk_pin + v * npad + lo, src[v] + lo, n * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaEventRecord(ctx->blk_ev[v], ctx->stream));
  }
  const cudaEvent_t* ev = ctx->blk_ev;
  const cudaError_t e = host_parallel(
      ctx->device, nout, staging_threads(nout * n * sizeof(double)), [&](int v) {
        const cudaError_t es = cudaEventSynchronize(ev[v]);
        if (es != cudaSuccess) return es;
        scatter(v);
        return cudaSuccess;
      });
  if (e != cudaSuccess) return fail_cuda(ctx, e, "block download");
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return B200BSSN_OK;
}

ConstraintArgs constraint_args(const b200bssn_plan* P, double* const* con,
                               const double* const* u, double* norms) {
  ConstraintArgs ca;
  std::memset(&ca, 0, sizeof(ca));
  for (int v = 0; v < kNumVars; ++v) ca.u[v] = u[v];
  for (int c = 0; c < kNumConstraints; ++c) ca.con[c] = con ? con[c] : nullptr;
  ca.norms = norms;
  ca.blocks = P->d_blocks;
  ca.units = P->d_units;
  ca.ranges = P->d_ranges;
  ca.cap = (int32_t)P->cap;
  ca.nslots = P->advective ? kNumDerivs + 3 * kNumVars : kNumDerivs;
  return ca;
}

}  // namespace

extern "C" {

int b200bssn_rhs(b200bssn_ctx* ctx, double* const* rhs, const double* const* u, uint32_t offset,
                 const double* pmin, const double* pmax, const uint32_t* sz, uint32_t bflag,
                 const b200bssn_params* prm) {
  b200bssn::host::NvtxRange nvtx_("b200bssn_rhs");
  const DropinCall call_;
  if (!ctx || !rhs || !u || !pmin || !pmax || !sz || !params_ok(prm))
    return B200BSSN_ERR_INVALID_ARGUMENT;
  for (int v = 0; v < kNumVars; ++v)
    if (!rhs[v] || !u[v]) return B200BSSN_ERR_INVALID_ARGUMENT;
  const double* ud[kNumVars];
  double* rd[kNumVars];
  int rc = prepare_block(ctx, u, offset, pmin, pmax, sz, bflag, prm->precision, ud, rd);
  if (rc != B200BSSN_OK) return rc;
  rc = launch_plan(ctx->blk_plan, rd, ud, prm, ctx->stream);
  if (rc != B200BSSN_OK) return rc;
  return copy_interior_back(ctx, rhs, rd, kNumVars, offset, sz);
}

int b200bssn_physical_constraints(b200bssn_ctx* ctx, double* const* con, const double* const* u,
                                  uint32_t offset, const double* pmin, const double* pmax,
                                  const uint32_t* sz, uint32_t bflag, uint32_t precision) {
  b200bssn::host::NvtxRange nvtx_("b200bssn_physical_constraints");
  const DropinCall call_;
  if (!ctx || !con || !u || !pmin || !pmax || !sz) return B200BSSN_ERR_INVALID_ARGUMENT;
  if (precision != B200BSSN_FP64 && precision != B200BSSN_MIXED) return B200BSSN_ERR_INVALID_ARGUMENT;
  for (int v = 0; v < kNumVars; ++v)
    if (!u[v]) return B200BSSN_ERR_INVALID_ARGUMENT;
  for (int c = 0; c < kNumConstraints; ++c)
    if (!con[c]) return B200BSSN_ERR_INVALID_ARGUMENT;
  const double* ud[kNumVars];
  double* rd[kNumVars];
  int rc = prepare_block(ctx, u, offset, pmin, pmax, sz, bflag, precision, ud, rd);
  if (rc != B200BSSN_OK) return rc;
  b200bssn_params prm;
  b200bssn_default_params(&prm);
  prm.precision = precision;
  const ConstraintArgs ca = constraint_args(ctx->blk_plan, rd, ud, nullptr);
  rc = launch_plan(ctx->blk_plan, rd, ud, &prm, ctx->stream, nullptr, &ca);
  if (rc != B200BSSN_OK) return rc;
  return copy_interior_back(ctx, con, rd, kNumConstraints, offset, sz);
}

int b200bssn_constraints_plan_device(b200bssn_plan* P, double* const* con_dev,
                                     const double* const* u_dev, double* block_norms_dev,
                                     void* stream) {
  b200bssn::host::NvtxRange nvtx_("b200bssn_constraints_plan_device");
  if (!P || !u_dev || (!con_dev && !block_norms_dev)) return B200BSSN_ERR_INVALID_ARGUMENT;
  for (int v = 0; v < kNumVars; ++v)
    if (!u_dev[v]) return B200BSSN_ERR_INVALID_ARGUMENT;
  if (con_dev)
    for (int c = 0; c < kNumConstraints; ++c)
      if (!con_dev[c]) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = P->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  if (block_norms_dev)
    CK(ctx, cudaMemsetAsync(block_norms_dev, 0,
                            P->blocks.size() * 2 * kNumConstraints * sizeof(double), s));
  b200bssn_params prm;
  b200bssn_default_params(&prm);
  prm.precision = P->precision;
  const ConstraintArgs ca = constraint_args(P, con_dev, u_dev, block_norms_dev);
  // the algebra arguments are unused on this path; u stands in for the rhs arrays
  return launch_plan(P, const_cast<double* const*>(u_dev), u_dev, &prm, s, nullptr, &ca);
}

int b200bssn_debug_block_scratch(b200bssn_ctx* ctx, double* slots, uint64_t npts) {
  if (!ctx || !slots || !ctx->blk_plan) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_plan* P = ctx->blk_plan;
  if (P->single_pass || P->chunks.size() != 1 || npts != P->points) return B200BSSN_ERR_INVALID_ARGUMENT;
  CK(ctx, cudaSetDevice(ctx->device));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  // the scratch is blocked by 32 points (scr_index): copy it whole, then gather
  const int ns = P->advective ? kNumDerivs + 3 * kNumVars : kNumDerivs;
  const size_t nd = (size_t)ns * P->cap;
  std::vector<double> d(nd), ko((size_t)kNumVars * P->cap);
  if (P->precision == B200BSSN_MIXED) {
    std::vector<float> tmp(nd);
    CK(ctx, cudaMemcpy(tmp.data(), P->dscr[0], nd * sizeof(float), cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < nd; ++k) d[k] = tmp[k];
  } else {
    CK(ctx, cudaMemcpy(d.data(), P->dscr[0], nd * sizeof(double), cudaMemcpyDeviceToHost));
  }
  if (P->precision == B200BSSN_MIXED) {
    std::vector<float> tmp(ko.size());
    CK(ctx, cudaMemcpy(tmp.data(), P->koscr[0], tmp.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < ko.size(); ++k) ko[k] = tmp[k];
  } else {
    CK(ctx, cudaMemcpy(ko.data(), P->koscr[0], ko.size() * sizeof(double), cudaMemcpyDeviceToHost));
  }
  auto at = [](int n, int s, uint64_t p) { return ((p >> 5) * n + s) * 32 + (p & 31); };
  for (int s = 0; s < kNumDerivs; ++s)
    for (uint64_t p = 0; p < npts; ++p) slots[s * npts + p] = d[at(ns, s, p)];
  for (int v = 0; v < kNumVars; ++v)
    for (uint64_t p = 0; p < npts; ++p) slots[(kNumDerivs + v) * npts + p] = ko[at(kNumVars, v, p)];
  return B200BSSN_OK;
}

}  // extern "C"
