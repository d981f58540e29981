/* b200bssn -- B200-native BSSN right-hand side for Dendro octree blocks.
 *
 * C ABI of the library (libb200bssn.so).  Plain pointers and sizes only.
 *
 * The reference interface this replaces is the per-block C++ entry point
 *
 *   void bssnrhs(double **uzipVarsRHS, const double **uZipVars,
 *                const unsigned int &offset, const double *ptmin, const double *ptmax,
 *                const unsigned int *sz, const unsigned int &bflag);
 *                                              (bssn/include/rhs.h:33-36,
 *                                               bssn/src/rhs.cpp:80-388)
 *
 * and the block loop around it, bssnRHS (bssn/src/rhs.cpp:7-70).  Variables are
 * the 24 BSSN fields in the reference's VAR order (bssn/include/grDef.h:31); each
 * block is sz[0]*sz[1]*sz[2] contiguous doubles at `offset` in every variable
 * array, x fastest (IDX(i,j,k) = i + nx*(j + ny*k), bssn/include/derivs.h:8), with
 * a 3-point ghost layer; ptmin/ptmax are the ghost-inclusive physical corners and
 * h = (ptmax-ptmin)/(sz-1) (bssn/src/rhs.cpp:144-146); bflag bits 0..5 mark the
 * faces LEFT,RIGHT,DOWN,UP,BACK,FRONT (bssn/include/def.h:13-18) that get
 * one-sided stencils and Sommerfeld values.  Only the interior [3,n-3)^3 of the
 * right-hand side is written.
 *
 * Every function returns 0 (B200BSSN_OK) or a negative error code; nothing
 * aborts the caller.  A context owns its CUDA stream and device buffers; calls on
 * one context must not overlap (use one context per host thread).
 */
#ifndef B200BSSN_H
#define B200BSSN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B200BSSN_NUM_VARS 24

enum b200bssn_status {
  B200BSSN_OK = 0,
  B200BSSN_ERR_INVALID_ARGUMENT = -1, /* null pointer, bad size, bad flag */
  B200BSSN_ERR_BLOCK_TOO_SMALL = -2,  /* an interior extent below 7 points */
  B200BSSN_ERR_CUDA = -3,             /* a CUDA runtime call failed; see b200bssn_last_error */
  B200BSSN_ERR_OUT_OF_MEMORY = -4,    /* device allocation failed */
  B200BSSN_ERR_NO_DEVICE = -5,        /* no usable sm_100 device */
  B200BSSN_ERR_NONFINITE = -6,        /* the NaN/Inf guard found a non-finite RHS value */
  B200BSSN_ERR_TIMEOUT = -7,          /* a bounded device wait gave up */
  B200BSSN_ERR_SIZE_LIMIT = -8        /* request exceeds a documented fixed limit */
};

/* Arithmetic of the per-point algebra. */
enum b200bssn_precision {
  B200BSSN_FP64 = 0,  /* everything in FP64 (the reference's arithmetic) */
  B200BSSN_MIXED = 1  /* FP64 state, FP64 stencils and KO, FP32 algebra */
};

/* What happens to the ghost points of the RHS arrays in the host batch call. */
enum b200bssn_ghost_policy {
  B200BSSN_GHOSTS_PRESERVE = 0, /* untouched, as the reference leaves them */
  B200BSSN_GHOSTS_ZERO = 1      /* set to 0 (Dendro's zip reads interior points only) */
};

/* Solver parameters: the bssn:: globals that bssnrhs reads
 * (bssn/src/parameters.cpp:99-109), plus the engine's own switches. */
typedef struct b200bssn_params {
  uint32_t lambda[4];      /* bssn::BSSN_LAMBDA                           */
  double lambda_f[2];      /* bssn::BSSN_LAMBDA_F                         */
  double eta_const;        /* bssn::ETA_CONST                             */
  double eta_r0;           /* bssn::ETA_R0                                */
  double eta_damping_exp;  /* bssn::ETA_DAMPING_EXP                       */
  double ko_sigma;         /* bssn::KO_DISS_SIGMA                         */
  uint32_t precision;      /* enum b200bssn_precision                     */
  uint32_t ghost_policy;   /* enum b200bssn_ghost_policy (host batch only) */
} b200bssn_params;

/* Fills `p` with the reference defaults (bssn/src/parameters.cpp:99-109). */
void b200bssn_default_params(b200bssn_params *p);

/* One octree block (the arguments bssnRHS derives from an ot::Block,
 * bssn/src/rhs.cpp:43-60). */
typedef struct b200bssn_block {
  uint64_t offset;   /* element offset of the block in every variable array */
  uint32_t sz[3];    /* padded extents, ghost layer of 3 included           */
  uint32_t bflag;    /* boundary face bits                                  */
  double pmin[3];    /* ghost-inclusive lower corner                        */
  double pmax[3];    /* ghost-inclusive upper corner                        */
} b200bssn_block;

typedef struct b200bssn_ctx b200bssn_ctx;
typedef struct b200bssn_plan b200bssn_plan;

/* Context on CUDA device `device` (its own non-blocking stream). */
int b200bssn_create(b200bssn_ctx **ctx, int device);
int b200bssn_destroy(b200bssn_ctx *ctx);
/* The context's stream as an opaque handle (a cudaStream_t). */
void *b200bssn_stream(b200bssn_ctx *ctx);
/* Text of the last CUDA error seen by this context (empty if none). */
const char *b200bssn_last_error(b200bssn_ctx *ctx);
const char *b200bssn_status_string(int status);

/* Drop-in for bssnrhs (bssn/include/rhs.h:33-36): one block, HOST arrays.
 * rhs[v] and u[v] (v < 24) are the caller's zipped arrays; the block's slice is
 * copied to the device, evaluated, and its interior copied back, both through a
 * pinned host buffer the context keeps (24 x the block's points, grown on
 * demand; host threads do the copies).  Blocks until the result is in `rhs`. */
int b200bssn_rhs(b200bssn_ctx *ctx, double *const *rhs, const double *const *u,
                 uint32_t offset, const double *pmin, const double *pmax,
                 const uint32_t *sz, uint32_t bflag, const b200bssn_params *prm);

/* Work plan for a fixed block list: descriptors, tiles and the derivative
 * scratch live on the device.  Build once, evaluate many times (RK stages).
 * `chunk_points` bounds the interior points evaluated per kernel pair (and so the
 * scratch: 1296 bytes per point in FP64, 648 in MIXED); 0 picks the default. */
int b200bssn_plan_create(b200bssn_ctx *ctx, const b200bssn_block *blocks, uint32_t nblocks,
                         uint32_t precision, uint64_t chunk_points, b200bssn_plan **plan);
int b200bssn_plan_destroy(b200bssn_plan *plan);

/* Tuning knobs of a plan (0 in any field: the default). */
typedef struct b200bssn_plan_options {
  uint64_t chunk_points;       /* interior points per kernel pair (scratch size) */
  uint32_t slab_depth;         /* max interior z planes per work unit (default 48) */
  uint32_t deriv_ctas_per_sm;  /* resident derivative CTAs per SM (default: as many as fit) */
  /* NULL, or one entry per block overriding slab_depth for that block (0: keep
   * slab_depth); lets a tuner pick the depth per block-size class. */
  const uint32_t *block_slab_depth;
  /* 0: the advective terms beta^i d_i use the centred 6th-order first derivatives, as
   * the reference's default (6th-order) build does (deriv64adv_* = deriv64_*,
   * bssn/src/derivs.cpp:2841-2881).  1: opt-in upwind mode -- they use the 4th-order
   * upwind stencils deriv42adv_* (bssn/src/derivs.cpp:495-900), upwinded by the sign
   * of the matching shift component; the scratch grows by 72 slots per point. */
  uint32_t advective;
  /* 1: a MIXED plan with centred advection evaluates the right-hand side (and RK4
   * stages) in one pass -- one persistent kernel over every block, its derivative
   * scratch in an L2-sized ring of tile-slab slots -- instead of the two-pass
   * kernels (derivative scratch through HBM).  FP64, the upwind mode, the
   * constraints and the host-array path always use the two-pass kernels. */
  uint32_t single_pass;
  /* Ring slots of the one-pass kernel (0: 128; each slot 3072 points, 2 MB). */
  uint32_t ring_slots;
  /* Tile height of the two-pass derivative kernels: 16 x tile_y columns per CTA, one
   * thread per column (0: 8; also 4 or 16). */
  uint32_t tile_y;
  /* Registers-per-thread split of the two-pass derivative kernels (the kinds without /
   * with second derivatives): 1 = 96 / 128 registers, 2 = 80 / 96 (one CTA per SM
   * more), 3 = 128 / 168 (one fewer); 2 and 3 with 16x8 tiles and centred advection
   * only.  0: the measured best -- 3 for FP64 with centred advection and 16x8 tiles,
   * else 1. */
  uint32_t deriv_regs;
  /* 2: the two-pass derivative kernels give each thread two output points (y pairs of
   * 16x16 tiles, CTAs of 128 threads), centred advection only; 0 or 1: one point. */
  uint32_t points_per_thread;
} b200bssn_plan_options;

/* b200bssn_plan_create with explicit options (opts may be NULL). */
int b200bssn_plan_create_ex(b200bssn_ctx *ctx, const b200bssn_block *blocks, uint32_t nblocks,
                            uint32_t precision, const b200bssn_plan_options *opts,
                            b200bssn_plan **plan);
/* Interior points covered by a plan, and the number of kernel launches one
 * evaluation issues. */
uint64_t b200bssn_plan_points(const b200bssn_plan *plan);
uint32_t b200bssn_plan_launches(const b200bssn_plan *plan);
/* 1 when the plan's right-hand side runs as the one-pass kernel, else 0. */
uint32_t b200bssn_plan_single_pass(const b200bssn_plan *plan);
/* Synchronises the context and reads the plan's device error word: B200BSSN_OK, or
 * B200BSSN_ERR_TIMEOUT when a bounded wait of the one-pass kernel ran out during
 * the last evaluation (its results are then incomplete). */
int b200bssn_plan_status(b200bssn_plan *plan);

/* Batched right-hand side on DEVICE arrays (the bssnRHS block loop,
 * bssn/src/rhs.cpp:41-68).  rhs_dev[v]/u_dev[v] are device pointers to the
 * zipped arrays.  Asynchronous on `stream` (NULL: the context stream); no
 * allocation, so it can be captured in a CUDA graph. prm->precision must match
 * the plan's. */
int b200bssn_rhs_plan_device(b200bssn_plan *plan, double *const *rhs_dev,
                             const double *const *u_dev, const b200bssn_params *prm,
                             void *stream);

/* Batched right-hand side on HOST arrays: uploads the plan's span of every
 * variable, evaluates, downloads the result (ghost handling per
 * prm->ghost_policy; PRESERVE brings back only each block's interior, so the
 * fastest transfers need page-locked host arrays).  `n_elems` is the length of
 * each host array.  Blocks until done. */
int b200bssn_rhs_plan_host(b200bssn_plan *plan, double *const *rhs, const double *const *u,
                           uint64_t n_elems, const b200bssn_params *prm);

/* ---- constraints --------------------------------------------------------- */

/* Number of constraint fields: ham, mom0, mom1, mom2 (VAR_CONSTRAINT C_HAM..C_MOM2,
 * bssn/include/grDef.h:40). */
#define B200BSSN_NUM_CONSTRAINTS 4

/* Drop-in for physical_constraints (bssn/CodeGen/physcon.cpp:12-15; expressions of
 * GR/constraints.py:166-177): one block, HOST arrays.  con[c] (c < 4: ham, mom0,
 * mom1, mom2) receive the constraints at the block's interior points; ghost points
 * are left untouched.  The reference's Psi4 outputs (C_PSI4_REAL/IMG) are not
 * computed.  The stencils use each axis' own spacing; the reference uses hx on all
 * three axes, which is the same on Dendro's cubic blocks.  `precision` selects
 * FP64 or split-precision stencils with FP32 algebra.  Blocks until done. */
int b200bssn_physical_constraints(b200bssn_ctx *ctx, double *const *con, const double *const *u,
                                  uint32_t offset, const double *pmin, const double *pmax,
                                  const uint32_t *sz, uint32_t bflag, uint32_t precision);

/* Constraints of every block of a plan on DEVICE arrays, in the plan's precision.
 * con_dev: NULL, or 4 device arrays indexed like u_dev, written at interior points.
 * block_norms_dev: NULL, or nblocks*8 device doubles, overwritten per block (plan
 * order) with { sum ham^2, sum mom0^2, sum mom1^2, sum mom2^2, max|ham|, max|mom0|,
 * max|mom1|, max|mom2| } over the block's interior points; a non-finite constraint
 * makes its maximum NaN.  At least one of the two must be given.  Asynchronous on
 * `stream` (NULL: the context stream); no allocation (graph-capturable). */
int b200bssn_constraints_plan_device(b200bssn_plan *plan, double *const *con_dev,
                                     const double *const *u_dev, double *block_norms_dev,
                                     void *stream);

/* ---- NaN/Inf guard ------------------------------------------------------- */

/* Scans the interior points of every block of the plan in `narrays` (1..24)
 * device arrays indexed like the state.  Returns B200BSSN_ERR_NONFINITE if any
 * value is NaN or infinite, with *first_bad (if non-NULL) the smallest offending
 * element index; B200BSSN_OK otherwise (*first_bad = UINT64_MAX).  Ghost points
 * are not scanned.  Synchronous on `stream` (NULL: the context stream). */
int b200bssn_check_finite(b200bssn_plan *plan, const double *const *arrays, uint32_t narrays,
                          uint64_t *first_bad, void *stream);

/* ---- RK4 time stepping ---------------------------------------------------- */

/* Classic 4-stage Runge-Kutta over a plan's blocks (BSSN_RK4_STAGES = 4,
 * bssn/include/parameters.h:37; the reference repository itself has no
 * integrator).  The stage update runs in the epilogue of the algebra kernel, in
 * FP64 in both precisions, so a stage is the plan's two launches per chunk and the
 * RHS never goes to memory.  The object owns three [24][span] FP64 buffers (the
 * accumulator and two stage states; span = the element range of the plan's
 * blocks).  Stage kernels write interior points only; ghost points of the stage
 * states keep what rk4_init (or the caller) put there, so a caller that exchanges
 * ghosts between blocks does it between stages, on the arrays rk4_stage_state
 * names.  Blocks with all six faces flagged (bflag 0x3F) never read ghosts. */
typedef struct b200bssn_rk4 b200bssn_rk4;

int b200bssn_rk4_create(b200bssn_plan *plan, b200bssn_rk4 **rk);
int b200bssn_rk4_destroy(b200bssn_rk4 *rk);
/* Copies u_dev's span (ghosts included) into both stage states.  Asynchronous. */
int b200bssn_rk4_init(b200bssn_rk4 *rk, const double *const *u_dev, void *stream);
/* Device arrays (24) holding the state that stage `stage` (0..3) reads; stage 0
 * reads the caller's u and reports NULL pointers. */
int b200bssn_rk4_stage_state(b200bssn_rk4 *rk, uint32_t stage, double **state);
/* One stage (0..3) of the step u_dev(t) -> u_dev(t + dt); the last stage updates
 * u_dev in place.  Asynchronous on `stream` (NULL: the context stream). */
int b200bssn_rk4_stage(b200bssn_rk4 *rk, uint32_t stage, double *const *u_dev, double dt,
                       const b200bssn_params *prm, void *stream);
/* The four stages back to back. */
int b200bssn_rk4_step(b200bssn_rk4 *rk, double *const *u_dev, double dt,
                      const b200bssn_params *prm, void *stream);
/* Captures `steps` (1..1000) full steps for fixed u_dev, dt and prm into a CUDA
 * graph owned by `rk` (replacing any earlier one); the capture itself runs nothing.
 * Synchronises the context stream first. */
int b200bssn_rk4_graph_capture(b200bssn_rk4 *rk, double *const *u_dev, double dt,
                               const b200bssn_params *prm, uint32_t steps);
/* Launches the captured graph on `stream` (NULL: the context stream). */
int b200bssn_rk4_graph_launch(b200bssn_rk4 *rk, void *stream);
/* Steps in the captured graph (0: none). */
uint32_t b200bssn_rk4_graph_steps(const b200bssn_rk4 *rk);

/* ---- allocation-free variant --------------------------------------------- */

/* Largest interior point count b200bssn_rhs_noalloc accepts: 32^3 (a 38^3
 * padded block).  Its fixed device array is 42.6 MB. */
#define B200BSSN_NOALLOC_MAX_POINTS 32768

/* The right-hand side of ONE block on DEVICE arrays without allocating any device
 * memory.  This entry point has no counterpart in the reference; it exists for
 * callers that cannot call cudaMalloc: frameworks whose pool allocator owns all of
 * the GPU's memory, and time-step loops that must avoid the device-wide
 * synchronisation cudaMalloc/cudaFree can cause.  The caller passes the inputs and
 * outputs (rhs_dev[v], u_dev[v]: device pointers, block at block->offset) and the
 * current device is used.  The derivative scratch and the work descriptors live in
 * one fixed device array inside the library (held by every GPU that loads it until
 * exit); blocks with more than B200BSSN_NOALLOC_MAX_POINTS interior points are
 * refused with B200BSSN_ERR_SIZE_LIMIT.  All calls share that array: calls that
 * overlap on the GPU race and corrupt each other, so serialise them per device.
 * The first call on a device looks up the array's address (cudaGetSymbolAddress)
 * and sets a kernel attribute with that device current; make it before any stream
 * capture.  That address is kept for the life of the process: calls after a
 * cudaDeviceReset of the device are not supported.  Asynchronous on `stream` (NULL:
 * the legacy default stream). */
int b200bssn_rhs_noalloc(double *const *rhs_dev, const double *const *u_dev,
                         const b200bssn_block *block, const b200bssn_params *prm,
                         void *stream);

/* ---- diagnostics ------------------------------------------------------- */

/* Evaluates the plan once on the context stream with CUDA events around each
 * launch and returns the summed device milliseconds of the derivative kernels
 * and of the algebra kernels.  Synchronous. */
int b200bssn_plan_profile(b200bssn_plan *plan, double *const *rhs_dev,
                          const double *const *u_dev, const b200bssn_params *prm,
                          double *ms_deriv, double *ms_algebra);

/* Copies the derivative scratch of the most recent b200bssn_rhs call on `ctx`
 * (one block, one chunk) to host `slots` [162][npts]: 138 derivatives, then 24 KO
 * sums, interior points x fastest.  For checking the stencil stage alone. */
int b200bssn_debug_block_scratch(b200bssn_ctx *ctx, double *slots, uint64_t npts);

/* Measured FMA throughput of `device` in TFLOP/s (an FMA counts 2 flops) for
 * FP64 (precision 0) or FP32 (precision 1): the roofline denominator of the
 * FP-pipe-bound algebra kernel. */
int b200bssn_fma_peak(int device, uint32_t precision, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* B200BSSN_H */
