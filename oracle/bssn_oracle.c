/* TEST INFRASTRUCTURE ONLY -- C restatement of the reference's bssnrhs path.
 *
 * Every operator below restates one routine of the reference:
 *   deriv64_x/_y/_z     bssn/src/derivs.cpp:2055-2434   (6th-order first derivative)
 *   deriv64_xx/_yy/_zz  bssn/src/derivs.cpp:2443-2833   (6th-order second derivative)
 *   ko_deriv42_x/_y/_z  bssn/src/derivs.cpp:915-1319    (Kreiss-Oliger, used at every order,
 *                                                        bssn/include/derivs.h:100)
 *   bssn_bcs            bssn/src/rhs.cpp:833-977        (Sommerfeld faces)
 *   bssnrhs             bssn/src/rhs.cpp:80-388         (orchestration)
 * The stencil tables hold the reference's coefficients in the reference's summation
 * order, and the scale factors are formed the same way, so with FMA contraction off
 * the stencils agree with the reference bit for bit; the algebra differs only by
 * its CSE (see bssn_oracle_algebra.c).
 */
#include "bssn_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NV BSSN_ORACLE_NUM_VARS

/* face bits, bssn/include/def.h:13-18 */
#define DIR_LEFT 0
#define DIR_RIGHT 1
#define DIR_DOWN 2
#define DIR_UP 3
#define DIR_BACK 4
#define DIR_FRONT 5

typedef struct { int off; double c; } tap_t;
typedef struct { int n; tap_t t[7]; } row_t;

/* One 1-D operator: the centred row (offsets from the point), the three rows of the
 * low-side closure (offsets from interior index 3) and of the high-side closure
 * (offsets from the last interior index n-4, i.e. ie-1). */
typedef struct {
  row_t centre;
  row_t lo[3];
  row_t hi[3];
} op1d_t;

/* deriv64_x centred row and 4th-order closures (derivs.cpp:2078-2155). */
static const op1d_t OP_D1 = {
    {6, {{-3, -1.0}, {-2, 9.0}, {-1, -45.0}, {1, 45.0}, {2, -9.0}, {3, 1.0}}},
    {{5, {{0, -25.0}, {1, 48.0}, {2, -36.0}, {3, 16.0}, {4, -3.0}}},
     {5, {{0, -3.0}, {1, -10.0}, {2, 18.0}, {3, -6.0}, {4, 1.0}}},
     {4, {{0, 1.0}, {1, -8.0}, {3, 8.0}, {4, -1.0}}}},
    {{4, {{-4, 1.0}, {-3, -8.0}, {-1, 8.0}, {0, -1.0}}},
     {5, {{-4, -1.0}, {-3, 6.0}, {-2, -18.0}, {-1, 10.0}, {0, 3.0}}},
     {5, {{-4, 3.0}, {-3, -16.0}, {-2, 36.0}, {-1, -48.0}, {0, 25.0}}}},
};

/* deriv64_xx centred row and closures (derivs.cpp:2469-2560). */
static const op1d_t OP_D2 = {
    {7, {{-3, 2.0}, {-2, -27.0}, {-1, 270.0}, {0, -490.0}, {1, 270.0}, {2, -27.0}, {3, 2.0}}},
    {{5, {{0, 35.0}, {1, -104.0}, {2, 114.0}, {3, -56.0}, {4, 11.0}}},
     {5, {{0, 11.0}, {1, -20.0}, {2, 6.0}, {3, 4.0}, {4, -1.0}}},
     {5, {{0, -1.0}, {1, 16.0}, {2, -30.0}, {3, 16.0}, {4, -1.0}}}},
    {{5, {{-4, -1.0}, {-3, 16.0}, {-2, -30.0}, {-1, 16.0}, {0, -1.0}}},
     {5, {{-4, -1.0}, {-3, 4.0}, {-2, 6.0}, {-1, -20.0}, {0, 11.0}}},
     {5, {{-4, 11.0}, {-3, -56.0}, {-2, 114.0}, {-1, -104.0}, {0, 35.0}}}},
};

/* ko_deriv42_x centred row and closures (derivs.cpp:942-1040); the low-side rows
 * are summed from the far point inwards, as the reference writes them. */
static const op1d_t OP_KO = {
    {7, {{-3, -1.0}, {-2, 6.0}, {-1, -15.0}, {0, 20.0}, {1, -15.0}, {2, 6.0}, {3, -1.0}}},
    {{4, {{3, 1.0}, {2, -3.0}, {1, 3.0}, {0, -1.0}}},
     {5, {{4, 1.0}, {3, -6.0}, {2, 12.0}, {1, -10.0}, {0, 3.0}}},
     {6, {{5, 1.0}, {4, -6.0}, {3, 15.0}, {2, -19.0}, {1, 12.0}, {0, -3.0}}}},
    {{6, {{-5, 1.0}, {-4, -6.0}, {-3, 15.0}, {-2, -19.0}, {-1, 12.0}, {0, -3.0}}},
     {5, {{-4, 1.0}, {-3, -6.0}, {-2, 12.0}, {-1, -10.0}, {0, 3.0}}},
     {4, {{-3, 1.0}, {-2, -3.0}, {-1, 3.0}, {0, -1.0}}}},
};

typedef enum { SCALE_MUL, SCALE_DIV } scale_kind_t;

typedef struct {
  double centre;            /* multiplies the centred sum */
  double lo[3], hi[3];      /* multiply or divide the closure sums */
  scale_kind_t closure_kind;
} scales_t;

static scales_t scales_d1(double h) {
  const double ih = 1.0 / h, by12 = ih / 12.0, by60 = ih / 60.0;
  scales_t s = {by60, {by12, by12, by12}, {by12, by12, by12}, SCALE_MUL};
  return s;
}

static scales_t scales_d2(double h) {
  const double ih2 = 1.0 / (h * h), by180 = ih2 / 180.0, by12 = ih2 / 12.0;
  scales_t s = {by180, {by12, by12, by12}, {by12, by12, by12}, SCALE_MUL};
  return s;
}

static scales_t scales_ko(double h) {
  const double pre = -1.0 / 64.0 / h;
  const double s3 = 59.0 / 48.0 * 64 * h, s2 = 43.0 / 48.0 * 64 * h, s1 = 49.0 / 48.0 * 64 * h;
  scales_t s = {pre, {s3, s2, s1}, {s1, s2, s3}, SCALE_DIV};
  return s;
}

static double row_sum(const row_t *r, const double *u, long base, long stride) {
  double acc = r->t[0].c * u[base + r->t[0].off * stride];
  for (int q = 1; q < r->n; ++q) acc += r->t[q].c * u[base + r->t[q].off * stride];
  return acc;
}

/* Apply `op` along `axis` at every point of the box lo..hi (hi exclusive); the
 * operator axis always spans the interior [3, n-3).  Closure rows replace the
 * centred row on the flagged faces, the high side last (the reference applies the
 * LEFT loop then the RIGHT loop). */
static void apply_axis(double *Du, const double *u, const unsigned int *sz, int axis,
                       const int *lo, const int *hi, const op1d_t *op, scales_t sc,
                       unsigned int bflag) {
  const long nx = sz[0], ny = sz[1];
  const long stride = axis == 0 ? 1 : (axis == 1 ? nx : nx * ny);
  const int n = (int)sz[axis];
  const int lo_face = (bflag >> (2 * axis)) & 1u;
  const int hi_face = (bflag >> (2 * axis + 1)) & 1u;
  for (int k = lo[2]; k < hi[2]; ++k)
    for (int j = lo[1]; j < hi[1]; ++j)
      for (int i = lo[0]; i < hi[0]; ++i) {
        const long pp = i + nx * (j + ny * (long)k);
        const int pos = axis == 0 ? i : (axis == 1 ? j : k);
        double val;
        if (hi_face && pos >= n - 6) {
          const int r = pos - (n - 6);
          const long base = pp + (long)((n - 4) - pos) * stride;
          const double s = row_sum(&op->hi[r], u, base, stride);
          val = sc.closure_kind == SCALE_MUL ? s * sc.hi[r] : s / sc.hi[r];
        } else if (lo_face && pos < 6) {
          const int r = pos - 3;
          const long base = pp - (long)(pos - 3) * stride;
          const double s = row_sum(&op->lo[r], u, base, stride);
          val = sc.closure_kind == SCALE_MUL ? s * sc.lo[r] : s / sc.lo[r];
        } else {
          val = row_sum(&op->centre, u, pp, stride) * sc.centre;
        }
        Du[pp] = val;
      }
}

static void box(int *lo, int *hi, const unsigned int *sz, int full_x, int full_y, int full_z) {
  lo[0] = full_x ? 0 : 3; hi[0] = full_x ? (int)sz[0] : (int)sz[0] - 3;
  lo[1] = full_y ? 0 : 3; hi[1] = full_y ? (int)sz[1] : (int)sz[1] - 3;
  lo[2] = full_z ? 0 : 3; hi[2] = full_z ? (int)sz[2] : (int)sz[2] - 3;
}

/* deriv64_x runs over all j,k (derivs.cpp:2067-2068: jb=kb=0) so that deriv64_y and
 * deriv64_z can be applied to its output; deriv64_y runs over all k (:2199,2202). */
void bssn_oracle_deriv64_x(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag) {
  int lo[3], hi[3];
  box(lo, hi, sz, 0, 1, 1);
  apply_axis(Du, u, sz, 0, lo, hi, &OP_D1, scales_d1(h), bflag);
}
void bssn_oracle_deriv64_y(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag) {
  int lo[3], hi[3];
  box(lo, hi, sz, 0, 0, 1);
  apply_axis(Du, u, sz, 1, lo, hi, &OP_D1, scales_d1(h), bflag);
}
void bssn_oracle_deriv64_z(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag) {
  int lo[3], hi[3];
  box(lo, hi, sz, 0, 0, 0);
  apply_axis(Du, u, sz, 2, lo, hi, &OP_D1, scales_d1(h), bflag);
}
void bssn_oracle_deriv64_xx(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag) {
  int lo[3], hi[3];
  box(lo, hi, sz, 0, 0, 0);
  apply_axis(Du, u, sz, 0, lo, hi, &OP_D2, scales_d2(h), bflag);
}
void bssn_oracle_deriv64_yy(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag) {
  int lo[3], hi[3];
  box(lo, hi, sz, 0, 0, 0);
  apply_axis(Du, u, sz, 1, lo, hi, &OP_D2, scales_d2(h), bflag);
}
void bssn_oracle_deriv64_zz(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag) {
  int lo[3], hi[3];
  box(lo, hi, sz, 0, 0, 0);
  apply_axis(Du, u, sz, 2, lo, hi, &OP_D2, scales_d2(h), bflag);
}
void bssn_oracle_ko_deriv42_x(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag) {
  int lo[3], hi[3];
  box(lo, hi, sz, 0, 0, 0);
  apply_axis(Du, u, sz, 0, lo, hi, &OP_KO, scales_ko(h), bflag);
}
void bssn_oracle_ko_deriv42_y(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag) {
  int lo[3], hi[3];
  box(lo, hi, sz, 0, 0, 0);
  apply_axis(Du, u, sz, 1, lo, hi, &OP_KO, scales_ko(h), bflag);
}
void bssn_oracle_ko_deriv42_z(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag) {
  int lo[3], hi[3];
  box(lo, hi, sz, 0, 0, 0);
  apply_axis(Du, u, sz, 2, lo, hi, &OP_KO, scales_ko(h), bflag);
}

/* ---- 4th-order upwind advective derivative, deriv42adv_x/_y/_z ---------------------
 * bssn/src/derivs.cpp:495-900 (the upwind operator of the reference's 4th-order build;
 * its 6th-order build wires deriv64adv_* to the centred deriv64_*, derivs.cpp:2841-2881).
 * At interior point i of the axis, with b = beta[pp]:
 *   centre      b > 0: (-3 u[i-1] - 10 u[i] + 18 u[i+1] - 6 u[i+2] + u[i+3]) / 12h
 *               else : (-u[i-3] + 6 u[i-2] - 18 u[i-1] + 10 u[i] + 3 u[i+1]) / 12h
 * and on a flagged low face (i = 3, 4, 5) / high face (i = n-6, n-5, n-4) the rows of
 * derivs.cpp:538-575 / 577-620 (second-order one-sided or centred rows / 2h, some of
 * them beta-dependent).  Rows are listed with offsets from i, in the reference's
 * summation order; scales multiply the row sums. */
typedef struct { row_t pos, neg; int half; } adv_row_t;  /* half: scale 1/2h, else 1/12h */

static const row_t ADV_C_POS = {5, {{-1, -3.0}, {0, -10.0}, {1, 18.0}, {2, -6.0}, {3, 1.0}}};
static const row_t ADV_C_NEG = {5, {{-3, -1.0}, {-2, 6.0}, {-1, -18.0}, {0, 10.0}, {1, 3.0}}};
static const row_t ADV_FWD2 = {3, {{0, -3.0}, {1, 4.0}, {2, -1.0}}};   /* (-3,4,-1)/2h */
static const row_t ADV_CEN2 = {2, {{-1, -1.0}, {1, 1.0}}};              /* (-1,0,1)/2h  */
static const row_t ADV_BWD2 = {3, {{-2, 1.0}, {-1, -4.0}, {0, 3.0}}};   /* (1,-4,3)/2h  */

/* low face rows i = 3, 4, 5 (derivs.cpp:538-575) and high face rows n-6, n-5, n-4
 * (derivs.cpp:577-620); `half` marks the /2h rows of each sign */
static const struct { const row_t *pos, *neg; int pos_half, neg_half; } ADV_LO[3] = {
    {&ADV_FWD2, &ADV_FWD2, 1, 1},
    {&ADV_FWD2, &ADV_CEN2, 1, 1},
    {&ADV_C_POS, &ADV_BWD2, 0, 1},
};
static const struct { const row_t *pos, *neg; int pos_half, neg_half; } ADV_HI[3] = {
    {&ADV_FWD2, &ADV_C_NEG, 1, 0},
    {&ADV_CEN2, &ADV_BWD2, 1, 1},
    {&ADV_BWD2, &ADV_BWD2, 1, 1},
};

static void apply_axis_adv(double *Du, const double *u, const double *beta, const unsigned int *sz,
                           int axis, double h, unsigned int bflag) {
  const long nx = sz[0], ny = sz[1];
  const long stride = axis == 0 ? 1 : (axis == 1 ? nx : nx * ny);
  const int n = (int)sz[axis];
  const int lo_face = (bflag >> (2 * axis)) & 1u;
  const int hi_face = (bflag >> (2 * axis + 1)) & 1u;
  const double ih = 1.0 / h, by2 = 0.50 * ih, by12 = ih / 12.0;  /* derivs.cpp:499-501 */
  for (int k = 3; k < (int)sz[2] - 3; ++k)
    for (int j = 3; j < (int)sz[1] - 3; ++j)
      for (int i = 3; i < (int)sz[0] - 3; ++i) {
        const long pp = i + nx * (j + ny * (long)k);
        const int pos = axis == 0 ? i : (axis == 1 ? j : k);
        const int up = beta[pp] > 0.0;
        const row_t *row = up ? &ADV_C_POS : &ADV_C_NEG;
        int half = 0;
        if (hi_face && pos >= n - 6) {
          const int r = pos - (n - 6);
          row = up ? ADV_HI[r].pos : ADV_HI[r].neg;
          half = up ? ADV_HI[r].pos_half : ADV_HI[r].neg_half;
        } else if (lo_face && pos < 6) {
          const int r = pos - 3;
          row = up ? ADV_LO[r].pos : ADV_LO[r].neg;
          half = up ? ADV_LO[r].pos_half : ADV_LO[r].neg_half;
        }
        Du[pp] = row_sum(row, u, pp, stride) * (half ? by2 : by12);
      }
}

void bssn_oracle_deriv42adv_x(double *Du, const double *u, double h, const unsigned int *sz,
                              const double *beta, unsigned int bflag) {
  apply_axis_adv(Du, u, beta, sz, 0, h, bflag);
}
void bssn_oracle_deriv42adv_y(double *Du, const double *u, double h, const unsigned int *sz,
                              const double *beta, unsigned int bflag) {
  apply_axis_adv(Du, u, beta, sz, 1, h, bflag);
}
void bssn_oracle_deriv42adv_z(double *Du, const double *u, double h, const unsigned int *sz,
                              const double *beta, unsigned int bflag) {
  apply_axis_adv(Du, u, beta, sz, 2, h, bflag);
}

/* Variables with second derivatives, in slot order (bssn/scripts/gen_bssnrhs_code:31-32),
 * given as VAR indices (bssn/include/grDef.h:31). */
static const int DD_VAR[11] = {12, 13, 14, 15, 16, 17, 1, 0, 6, 7, 8};

/* Sommerfeld falloff and asymptotic value per VAR index (bssn/src/rhs.cpp:261-320). */
static const double BC_FALLOFF[NV] = {1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1,
                                      1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2};
static const double BC_ASYMP[NV] = {1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                    1, 0, 0, 1, 0, 1, 0, 0, 0, 0, 0, 0};

/* Compute the 138 derivative arrays of a block (each npad long) the way
 * bssn/scripts/bssnrhs_derivs.h calls the stencils:  d[3v+a] = grad_a_<v>,
 * d[72 + 6q + m] = grad2_<pair m>_<DD_VAR[q]>.  Mixed pairs are compositions:
 * (0,1)=D_y(D_x u), (0,2)=D_z(D_x u), (1,2)=D_z(D_y u). */
static void all_derivatives(double **d, const double *const *u, unsigned int offset,
                            const double *h, const unsigned int *sz, unsigned int bflag) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int v = 0; v < NV; ++v) {
    const double *f = u[v] + offset;
    bssn_oracle_deriv64_x(d[3 * v + 0], f, h[0], sz, bflag);
    bssn_oracle_deriv64_y(d[3 * v + 1], f, h[1], sz, bflag);
    bssn_oracle_deriv64_z(d[3 * v + 2], f, h[2], sz, bflag);
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < 11; ++q) {
    const int v = DD_VAR[q];
    const double *f = u[v] + offset;
    double **g = d + 72 + 6 * q;
    bssn_oracle_deriv64_xx(g[0], f, h[0], sz, bflag);
    bssn_oracle_deriv64_y(g[1], d[3 * v + 0], h[1], sz, bflag);
    bssn_oracle_deriv64_z(g[2], d[3 * v + 0], h[2], sz, bflag);
    bssn_oracle_deriv64_yy(g[3], f, h[1], sz, bflag);
    bssn_oracle_deriv64_z(g[4], d[3 * v + 1], h[2], sz, bflag);
    bssn_oracle_deriv64_zz(g[5], f, h[2], sz, bflag);
  }
}

static void ko_sums(double **ko, const double *const *u, unsigned int offset, const double *h,
                    const unsigned int *sz, unsigned int bflag) {
  const long npad = (long)sz[0] * sz[1] * sz[2];
#pragma omp parallel for schedule(dynamic, 1)
  for (int v = 0; v < NV; ++v) {
    double *kx = (double *)calloc(npad, sizeof(double));
    double *ky = (double *)calloc(npad, sizeof(double));
    double *kz = (double *)calloc(npad, sizeof(double));
    const double *f = u[v] + offset;
    bssn_oracle_ko_deriv42_x(kx, f, h[0], sz, bflag);
    bssn_oracle_ko_deriv42_y(ky, f, h[1], sz, bflag);
    bssn_oracle_ko_deriv42_z(kz, f, h[2], sz, bflag);
    /* rhs.cpp:332-369 adds sigma*(grad_0 + grad_1 + grad_2): keep that sum order */
    for (long p = 0; p < npad; ++p) ko[v][p] = kx[p] + ky[p] + kz[p];
    free(kx); free(ky); free(kz);
  }
}

static double **alloc_arrays(int n, long npad) {
  double **a = (double **)malloc(sizeof(double *) * n);
  for (int s = 0; s < n; ++s) a[s] = (double *)calloc(npad, sizeof(double));
  return a;
}

static void free_arrays(double **a, int n) {
  for (int s = 0; s < n; ++s) free(a[s]);
  free(a);
}

#define NADV (BSSN_ORACLE_NUM_DERIVS + 3 * NV)  /* derivative slots of the upwind mode */

static void oracle_rhs_impl(double *const *rhs, const double *const *u, unsigned int offset,
                            const double *pmin, const double *pmax, const unsigned int *sz,
                            unsigned int bflag, const bssn_oracle_params *prm, int advective) {
  const int nx = (int)sz[0], ny = (int)sz[1], nz = (int)sz[2];
  const long npad = (long)nx * ny * nz;
  const double h[3] = {(pmax[0] - pmin[0]) / (nx - 1), (pmax[1] - pmin[1]) / (ny - 1),
                       (pmax[2] - pmin[2]) / (nz - 1)};
  const int nslots = advective ? NADV : BSSN_ORACLE_NUM_DERIVS;
  double **d = alloc_arrays(nslots, npad);
  all_derivatives(d, u, offset, h, sz, bflag);
  if (advective) {
    /* agrad_a_<v> = adv_deriv_a(<v>, beta_a) as bssn/scripts/bssnrhs_derivs_adv.h calls it */
#pragma omp parallel for schedule(dynamic, 1)
    for (int v = 0; v < NV; ++v) {
      const double *f = u[v] + offset;
      double **g = d + BSSN_ORACLE_NUM_DERIVS + 3 * v;
      bssn_oracle_deriv42adv_x(g[0], f, h[0], sz, u[6] + offset, bflag);
      bssn_oracle_deriv42adv_y(g[1], f, h[1], sz, u[7] + offset, bflag);
      bssn_oracle_deriv42adv_z(g[2], f, h[2], sz, u[8] + offset, bflag);
    }
  }

  const double par[6] = {(double)prm->lambda[0], (double)prm->lambda[1], (double)prm->lambda[2],
                         (double)prm->lambda[3], prm->lambda_f[0],       prm->lambda_f[1]};
  /* interior algebra loop, rhs.cpp:206-258 */
#pragma omp parallel for schedule(static)
  for (int k = 3; k < nz - 3; ++k) {
    const double z = pmin[2] + k * h[2];
    double uv[NV], dv[NADV], out[NV];
    for (int j = 3; j < ny - 3; ++j) {
      const double y = pmin[1] + j * h[1];
      for (int i = 3; i < nx - 3; ++i) {
        const double x = pmin[0] + i * h[0];
        const long pp = i + (long)nx * (j + (long)ny * k);
        const double r = sqrt(x * x + y * y + z * z);
        double eta = prm->eta_const;
        if (r >= prm->eta_r0) eta *= pow(prm->eta_r0 / r, prm->eta_damping_exp);
        for (int v = 0; v < NV; ++v) uv[v] = u[v][offset + pp];
        for (int s = 0; s < nslots; ++s) dv[s] = d[s][pp];
        if (advective)
          bssn_oracle_algebra_adv(uv, dv, par, eta, out);
        else
          bssn_oracle_algebra(uv, dv, par, eta, out);
        for (int v = 0; v < NV; ++v) rhs[v][offset + pp] = out[v];
      }
    }
  }

  /* Sommerfeld faces, rhs.cpp:261-320 -> bssn_bcs (rhs.cpp:833-977) */
  if (bflag != 0) {
    for (int v = 0; v < NV; ++v) {
      for (int face = 0; face < 6; ++face) {
        if (!(bflag & (1u << face))) continue;
        const int axis = face / 2;
        const int plane = (face & 1) ? (int)sz[axis] - 4 : 3;
        int lo[3] = {3, 3, 3}, hi[3] = {nx - 3, ny - 3, nz - 3};
        lo[axis] = plane;
        hi[axis] = plane + 1;
        for (int k = lo[2]; k < hi[2]; ++k)
          for (int j = lo[1]; j < hi[1]; ++j)
            for (int i = lo[0]; i < hi[0]; ++i) {
              const double x = pmin[0] + i * h[0];
              const double y = pmin[1] + j * h[1];
              const double z = pmin[2] + k * h[2];
              const long pp = i + (long)nx * (j + (long)ny * k);
              const double inv_r = 1.0 / sqrt(x * x + y * y + z * z);
              rhs[v][offset + pp] =
                  -inv_r * (x * d[3 * v][pp] + y * d[3 * v + 1][pp] + z * d[3 * v + 2][pp] +
                            BC_FALLOFF[v] * (u[v][offset + pp] - BC_ASYMP[v]));
            }
      }
    }
  }

  /* KO dissipation, rhs.cpp:323-369: after the boundary values are in place */
  double **ko = alloc_arrays(NV, npad);
  ko_sums(ko, u, offset, h, sz, bflag);
  const double sigma = prm->ko_sigma;
#pragma omp parallel for schedule(static)
  for (int k = 3; k < nz - 3; ++k)
    for (int j = 3; j < ny - 3; ++j)
      for (int i = 3; i < nx - 3; ++i) {
        const long pp = i + (long)nx * (j + (long)ny * k);
        for (int v = 0; v < NV; ++v) rhs[v][offset + pp] += sigma * ko[v][pp];
      }
  free_arrays(ko, NV);
  free_arrays(d, nslots);
}

void bssn_oracle_rhs(double *const *rhs, const double *const *u, unsigned int offset,
                     const double *pmin, const double *pmax, const unsigned int *sz,
                     unsigned int bflag, const bssn_oracle_params *prm) {
  oracle_rhs_impl(rhs, u, offset, pmin, pmax, sz, bflag, prm, 0);
}

void bssn_oracle_rhs_adv(double *const *rhs, const double *const *u, unsigned int offset,
                         const double *pmin, const double *pmax, const unsigned int *sz,
                         unsigned int bflag, const bssn_oracle_params *prm) {
  oracle_rhs_impl(rhs, u, offset, pmin, pmax, sz, bflag, prm, 1);
}

void bssn_oracle_derivative_slots(double *slots, const double *const *u, unsigned int offset,
                                  const double *pmin, const double *pmax,
                                  const unsigned int *sz, unsigned int bflag) {
  const int nx = (int)sz[0], ny = (int)sz[1], nz = (int)sz[2];
  const long npad = (long)nx * ny * nz;
  const int I0 = nx - 6, I1 = ny - 6, I2 = nz - 6;
  const long npts = (long)I0 * I1 * I2;
  const double h[3] = {(pmax[0] - pmin[0]) / (nx - 1), (pmax[1] - pmin[1]) / (ny - 1),
                       (pmax[2] - pmin[2]) / (nz - 1)};
  double **d = alloc_arrays(BSSN_ORACLE_NUM_DERIVS, npad);
  double **ko = alloc_arrays(NV, npad);
  all_derivatives(d, u, offset, h, sz, bflag);
  ko_sums(ko, u, offset, h, sz, bflag);
  for (int k = 3; k < nz - 3; ++k)
    for (int j = 3; j < ny - 3; ++j)
      for (int i = 3; i < nx - 3; ++i) {
        const long pp = i + (long)nx * (j + (long)ny * k);
        const long p = (i - 3) + (long)I0 * ((j - 3) + (long)I1 * (k - 3));
        for (int s = 0; s < BSSN_ORACLE_NUM_DERIVS; ++s) slots[s * npts + p] = d[s][pp];
        for (int v = 0; v < NV; ++v) slots[(BSSN_ORACLE_NUM_DERIVS + v) * npts + p] = ko[v][pp];
      }
  free_arrays(ko, NV);
  free_arrays(d, BSSN_ORACLE_NUM_DERIVS);
}

/* Hamiltonian and momentum constraints (GR/constraints.py:166-177) at the interior
 * points of one block, from the derivative arrays bssnrhs materialises. */
void bssn_oracle_block_constraints(double *const *con, const double *const *u, unsigned int offset,
                                   const double *pmin, const double *pmax,
                                   const unsigned int *sz, unsigned int bflag) {
  const int nx = (int)sz[0], ny = (int)sz[1], nz = (int)sz[2];
  const long npad = (long)nx * ny * nz;
  const double h[3] = {(pmax[0] - pmin[0]) / (nx - 1), (pmax[1] - pmin[1]) / (ny - 1),
                       (pmax[2] - pmin[2]) / (nz - 1)};
  double **d = alloc_arrays(BSSN_ORACLE_NUM_DERIVS, npad);
  all_derivatives(d, u, offset, h, sz, bflag);
#pragma omp parallel for schedule(static)
  for (int k = 3; k < nz - 3; ++k) {
    double uv[NV], dv[BSSN_ORACLE_NUM_DERIVS], out[4];
    for (int j = 3; j < ny - 3; ++j)
      for (int i = 3; i < nx - 3; ++i) {
        const long pp = i + (long)nx * (j + (long)ny * k);
        for (int v = 0; v < NV; ++v) uv[v] = u[v][offset + pp];
        for (int s = 0; s < BSSN_ORACLE_NUM_DERIVS; ++s) dv[s] = d[s][pp];
        bssn_oracle_constraints(uv, dv, out);
        for (int c = 0; c < 4; ++c) con[c][offset + pp] = out[c];
      }
  }
  free_arrays(d, BSSN_ORACLE_NUM_DERIVS);
}
