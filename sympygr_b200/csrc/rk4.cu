// Classic RK4 time stepping of a plan's blocks on the device, with the stage
// update fused into the algebra kernel (RkStage in plan_types.h) and whole steps
// captured as CUDA graphs.
//
// The reference repository has no time integrator (Dendro's RK loop lives outside
// it; bssn/include/parameters.h:37 fixes BSSN_RK4_STAGES = 4).  Stage s reads the
// state S_s and writes S_{s+1}:
//   S_0 = u^n (the caller's arrays)   -> S_1 in buffer A, acc  = dt/6 k1
//   S_1 = A                           -> S_2 in buffer B, acc += dt/3 k2
//   S_2 = B                           -> S_3 in buffer A, acc += dt/3 k3
//   S_3 = A                           -> u^{n+1} = u^n + acc + dt/6 k4 in place
// Each buffer is [24][span] over the element range the plan's blocks touch; the
// stage kernels write interior points only.  Ghost points of A and B hold whatever
// b200bssn_rk4_init (or the caller, through b200bssn_rk4_stage_state) put there:
// Dendro refreshes them between stages by its unzip exchange, which is outside
// this library; blocks with all six faces flagged never read them.
#include <cuda_runtime.h>

#include <cstring>

#include "b200bssn.h"
#include "plan_internal.h"
#include "plan_types.h"

using namespace b200bssn;
using b200bssn::host::fail_cuda;
using b200bssn::host::launch_plan;
using b200bssn::host::params_ok;

#define CK B200BSSN_CK

struct b200bssn_rk4 {
  b200bssn_plan* plan = nullptr;
  uint64_t lo = 0, len = 0;
  double* buf = nullptr;  // acc | A | B, each [24][len]
  double* acc[kNumVars];
  double* sa[kNumVars];
  double* sb[kNumVars];
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint32_t graph_steps = 0;
};

namespace {

void release_graph(b200bssn_rk4* R) {
  if (R->exec) cudaGraphExecDestroy(R->exec);
  if (R->graph) cudaGraphDestroy(R->graph);
  R->exec = nullptr;
  R->graph = nullptr;
  R->graph_steps = 0;
}

bool ptrs_ok(const double* const* p) {
  if (!p) return false;
  for (int v = 0; v < kNumVars; ++v)
    if (!p[v]) return false;
  return true;
}

int enqueue_stage(b200bssn_rk4* R, uint32_t stage, double* const* u, double dt,
                  const b200bssn_params* prm, cudaStream_t s) {
  static const double kW[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
  static const double kC[4] = {0.5, 0.5, 1.0, 0.0};
  RkStage rk;
  std::memset(&rk, 0, sizeof(rk));
  rk.mode = stage == 0 ? RK_FIRST : (stage == 3 ? RK_LAST : RK_MIDDLE);
  rk.w = dt * kW[stage];
  rk.c = dt * kC[stage];
  const double* in[kNumVars];
  for (int v = 0; v < kNumVars; ++v) {
    rk.acc[v] = R->acc[v];
    rk.base[v] = u[v];
    rk.next[v] = stage == 1 ? R->sb[v] : R->sa[v];
    in[v] = stage == 0 ? u[v] : (stage == 2 ? R->sb[v] : R->sa[v]);
  }
  // the RHS pointers are unused in a stage; the stage state stands in for them
  return launch_plan(R->plan, const_cast<double* const*>(in), in, prm, s, nullptr, nullptr, &rk);
}

int enqueue_step(b200bssn_rk4* R, double* const* u, double dt, const b200bssn_params* prm,
                 cudaStream_t s) {
  for (uint32_t st = 0; st < 4; ++st) {
    const int rc = enqueue_stage(R, st, u, dt, prm, s);
    if (rc != B200BSSN_OK) return rc;
  }
  return B200BSSN_OK;
}

bool step_args_ok(const b200bssn_rk4* R, double* const* u, double dt, const b200bssn_params* prm) {
  return R && ptrs_ok(u) && params_ok(prm) && prm->precision == R->plan->precision && dt > 0.0 &&
         dt < 1e300;
}

}  // namespace

extern "C" {

int b200bssn_rk4_create(b200bssn_plan* plan, b200bssn_rk4** out) {
  if (!plan || !out) return B200BSSN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  b200bssn_ctx* ctx = plan->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  b200bssn_rk4* R = new b200bssn_rk4();
  R->plan = plan;
  R->lo = plan->span_lo;
  R->len = plan->span_hi - plan->span_lo;
  const size_t per = (size_t)kNumVars * R->len;
  cudaError_t e = cudaMalloc((void**)&R->buf, 3 * per * sizeof(double));
  if (e != cudaSuccess) {
    delete R;
    return fail_cuda(ctx, e, "rk4 buffers");
  }
  for (int v = 0; v < kNumVars; ++v) {
    // shifted so that element index `lo` of a variable lands at its slice start
    R->acc[v] = R->buf + (size_t)v * R->len - R->lo;
    R->sa[v] = R->buf + per + (size_t)v * R->len - R->lo;
    R->sb[v] = R->buf + 2 * per + (size_t)v * R->len - R->lo;
  }
  *out = R;
  return B200BSSN_OK;
}

int b200bssn_rk4_destroy(b200bssn_rk4* R) {
  if (!R) return B200BSSN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(R->plan->ctx->device);
  cudaStreamSynchronize(R->plan->ctx->stream);
  release_graph(R);
  cudaFree(R->buf);
  delete R;
  return B200BSSN_OK;
}

int b200bssn_rk4_init(b200bssn_rk4* R, const double* const* u_dev, void* stream) {
  if (!R || !ptrs_ok(u_dev)) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = R->plan->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  const size_t bytes = R->len * sizeof(double);
  for (int v = 0; v < kNumVars; ++v) {
    CK(ctx, cudaMemcpyAsync(R->sa[v] + R->lo, u_dev[v] + R->lo, bytes, cudaMemcpyDeviceToDevice, s));
    CK(ctx, cudaMemcpyAsync(R->sb[v] + R->lo, u_dev[v] + R->lo, bytes, cudaMemcpyDeviceToDevice, s));
  }
  return B200BSSN_OK;
}

int b200bssn_rk4_stage_state(b200bssn_rk4* R, uint32_t stage, double** state) {
  if (!R || !state || stage > 3) return B200BSSN_ERR_INVALID_ARGUMENT;
  for (int v = 0; v < kNumVars; ++v)
    state[v] = stage == 0 ? nullptr : (stage == 2 ? R->sb[v] : R->sa[v]);
  return B200BSSN_OK;
}

int b200bssn_rk4_stage(b200bssn_rk4* R, uint32_t stage, double* const* u_dev, double dt,
                       const b200bssn_params* prm, void* stream) {
  b200bssn::host::NvtxRange nvtx_("b200bssn_rk4_stage");
  if (!step_args_ok(R, u_dev, dt, prm) || stage > 3) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = R->plan->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  return enqueue_stage(R, stage, u_dev, dt, prm, stream ? (cudaStream_t)stream : ctx->stream);
}

int b200bssn_rk4_step(b200bssn_rk4* R, double* const* u_dev, double dt,
                      const b200bssn_params* prm, void* stream) {
  b200bssn::host::NvtxRange nvtx_("b200bssn_rk4_step");
  if (!step_args_ok(R, u_dev, dt, prm)) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = R->plan->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  return enqueue_step(R, u_dev, dt, prm, stream ? (cudaStream_t)stream : ctx->stream);
}

int b200bssn_rk4_graph_capture(b200bssn_rk4* R, double* const* u_dev, double dt,
                               const b200bssn_params* prm, uint32_t steps) {
  if (!step_args_ok(R, u_dev, dt, prm) || steps == 0 || steps > 1000)
    return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = R->plan->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  release_graph(R);
  CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int rc = B200BSSN_OK;
  for (uint32_t i = 0; i < steps && rc == B200BSSN_OK; ++i)
    rc = enqueue_step(R, u_dev, dt, prm, ctx->stream);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (rc != B200BSSN_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail_cuda(ctx, e, "rk4 graph capture");
  R->graph = g;
  const cudaError_t ei = cudaGraphInstantiate(&R->exec, g, 0);
  if (ei != cudaSuccess) {
    release_graph(R);
    return fail_cuda(ctx, ei, "rk4 graph instantiate");
  }
  R->graph_steps = steps;
  return B200BSSN_OK;
}

int b200bssn_rk4_graph_launch(b200bssn_rk4* R, void* stream) {
  b200bssn::host::NvtxRange nvtx_("b200bssn_rk4_graph_launch");
  if (!R || !R->exec) return B200BSSN_ERR_INVALID_ARGUMENT;
  b200bssn_ctx* ctx = R->plan->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  CK(ctx, cudaGraphLaunch(R->exec, stream ? (cudaStream_t)stream : ctx->stream));
  return B200BSSN_OK;
}

uint32_t b200bssn_rk4_graph_steps(const b200bssn_rk4* R) { return R ? R->graph_steps : 0; }

}  // extern "C"
