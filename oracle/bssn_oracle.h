/* TEST INFRASTRUCTURE ONLY -- the oracle for the BSSN right-hand side.
 *
 * A C restatement of the reference's CPU path `bssnrhs`
 * (bssn/src/rhs.cpp:80-388) in its default build (6th-order centred stencils,
 * bssn/CMakeLists.txt:62 and bssn/include/derivs.h:87-100; KO dissipation from the
 * 4th-order family; centred "advective" derivatives, bssn/src/derivs.cpp:2841-2881).
 * It is pinned against the reference itself (compiled into oracle/_ref by the
 * Makefile) and against golden fixtures in tests/golden/.  Only tests, the smoke
 * check and the CPU-baseline leg of bench.py use it; the product never does.
 */
#ifndef BSSN_ORACLE_H
#define BSSN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define BSSN_ORACLE_NUM_VARS 24
#define BSSN_ORACLE_NUM_DERIVS 138   /* 72 first + 66 second (algebra inputs) */
#define BSSN_ORACLE_NUM_SLOTS 162    /* + 24 KO sums */

typedef struct {
  unsigned int lambda[4];   /* bssn::BSSN_LAMBDA   (bssn/src/parameters.cpp:99)  */
  double lambda_f[2];       /* bssn::BSSN_LAMBDA_F (:100)                         */
  double eta_const;         /* bssn::ETA_CONST     (:102)                         */
  double eta_r0;            /* bssn::ETA_R0        (:103)                         */
  double eta_damping_exp;   /* bssn::ETA_DAMPING_EXP (:105)                       */
  double ko_sigma;          /* bssn::KO_DISS_SIGMA (:107)                         */
} bssn_oracle_params;

/* Derivative operators on one padded block (layout IDX(i,j,k)=i+nx*(j+ny*k),
 * bssn/include/derivs.h:8).  Each writes exactly the points the reference
 * routine writes and leaves the rest of `Du` untouched. */
void bssn_oracle_deriv64_x(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag);
void bssn_oracle_deriv64_y(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag);
void bssn_oracle_deriv64_z(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag);
void bssn_oracle_deriv64_xx(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag);
void bssn_oracle_deriv64_yy(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag);
void bssn_oracle_deriv64_zz(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag);
void bssn_oracle_ko_deriv42_x(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag);
void bssn_oracle_ko_deriv42_y(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag);
void bssn_oracle_ko_deriv42_z(double *Du, const double *u, double h, const unsigned int *sz, unsigned int bflag);

/* 4th-order upwind advective derivatives (bssn/src/derivs.cpp:495-900): interior
 * points only, upwinded by the sign of beta[pp] (the matching shift component). */
void bssn_oracle_deriv42adv_x(double *Du, const double *u, double h, const unsigned int *sz,
                              const double *beta, unsigned int bflag);
void bssn_oracle_deriv42adv_y(double *Du, const double *u, double h, const unsigned int *sz,
                              const double *beta, unsigned int bflag);
void bssn_oracle_deriv42adv_z(double *Du, const double *u, double h, const unsigned int *sz,
                              const double *beta, unsigned int bflag);

/* Per-point algebra (generated; oracle/bssn_oracle_algebra.c). */
void bssn_oracle_algebra(const double *u, const double *d, const double *par, double eta, double *out);

/* The same with the advective derivatives in their own slots d[138 + 3v + a]
 * (generated; oracle/bssn_oracle_algebra_adv.c). */
void bssn_oracle_algebra_adv(const double *u, const double *d, const double *par, double eta,
                             double *out);

/* Per-point Hamiltonian and momentum constraints (generated;
 * oracle/bssn_oracle_constraints.c): out[4] = ham, mom0, mom1, mom2. */
void bssn_oracle_constraints(const double *u, const double *d, double *out);

/* Constraints of one block at its interior points: con[c][offset + IDX] for c < 4
 * (ham, mom0..2), computed from the same derivatives bssnrhs uses. */
void bssn_oracle_block_constraints(double *const *con, const double *const *u, unsigned int offset,
                                   const double *pmin, const double *pmax,
                                   const unsigned int *sz, unsigned int bflag);

/* Whole-block right-hand side with the reference's signature semantics
 * (bssn/include/rhs.h:33-36): reads u[v][offset + IDX], writes the interior
 * [3,n-3)^3 of rhs[v][offset + IDX]; ghosts of rhs are not touched. */
void bssn_oracle_rhs(double *const *rhs, const double *const *u, unsigned int offset,
                     const double *pmin, const double *pmax, const unsigned int *sz,
                     unsigned int bflag, const bssn_oracle_params *prm);

/* bssn_oracle_rhs in the opt-in upwind mode: the advective terms beta^i d_i f use the
 * 4th-order upwind derivatives above instead of the centred 6th-order ones. */
void bssn_oracle_rhs_adv(double *const *rhs, const double *const *u, unsigned int offset,
                         const double *pmin, const double *pmax, const unsigned int *sz,
                         unsigned int bflag, const bssn_oracle_params *prm);

/* The 162 derivative slots of one block at its interior points, compact
 * ordering p = (i-3) + I0*((j-3) + I1*(k-3)); slots[s*npts + p].  Slots
 * 0..137 follow the algebra's input table, 138..161 are KO sums per variable. */
void bssn_oracle_derivative_slots(double *slots, const double *const *u, unsigned int offset,
                                  const double *pmin, const double *pmax,
                                  const unsigned int *sz, unsigned int bflag);

#ifdef __cplusplus
}
#endif
#endif
