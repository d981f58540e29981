// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// C-ABI wrapper around the reference's own CPU `bssnrhs`
// (bssn/src/rhs.cpp:80-388, declared at bssn/include/rhs.h:33-36), compiled from
// the reference sources by oracle/Makefile into oracle/_ref/. The tests use it to
// pin the C restatement in oracle/bssn_oracle.c and to produce golden fixtures; the
// benchmark's reference arm times `ref_bssnrhs_blocks_omp` on the host cores.
#include <omp.h>
#include <cstring>
#include "rhs.h"

// The reference's generated constraint evaluator (bssn/CodeGen/physcon.cpp:12-15),
// compiled unmodified against the declarations in oracle/ref_shim/physcon.h.
void physical_constraints(double **uZipConVars, const double **uZipVars, const unsigned int &offset,
                          const double *pmin, const double *pmax, const unsigned int *sz,
                          const unsigned int &bflag);

extern "C" {

// Sets the bssn:: globals that bssnrhs reads (bssn/src/parameters.cpp:99-109).
void ref_set_params(const unsigned int* lambda, const double* lambda_f, double eta_const,
                    double eta_r0, double eta_damping_exp, double ko_sigma) {
  for (int i = 0; i < 4; ++i) bssn::BSSN_LAMBDA[i] = lambda[i];
  bssn::BSSN_LAMBDA_F[0] = lambda_f[0];
  bssn::BSSN_LAMBDA_F[1] = lambda_f[1];
  bssn::ETA_CONST = eta_const;
  bssn::ETA_R0 = eta_r0;
  bssn::ETA_DAMPING_EXP = eta_damping_exp;
  bssn::KO_DISS_SIGMA = ko_sigma;
}

// One block through the reference entry point, exactly as the Dendro block loop
// calls it (bssn/src/rhs.cpp:63-66).
void ref_bssnrhs(double** rhs, const double** u, unsigned int offset, const double* pmin,
                 const double* pmax, const unsigned int* sz, unsigned int bflag) {
  bssnrhs(rhs, u, offset, pmin, pmax, sz, bflag);
}

// The reference's staged variant (bssn/src/rhs.cpp:392-825, selected by
// BSSN_RHS_STAGED_COMP in bssnRHS): the same right-hand side evaluated one
// equation group at a time.
void ref_bssnrhs_sep(double** rhs, const double** u, unsigned int offset, const double* pmin,
                     const double* pmax, const unsigned int* sz, unsigned int bflag) {
  bssnrhs_sep(rhs, u, offset, pmin, pmax, sz, bflag);
}

// Block list through the reference's block-parallel OpenMP loop
// (bssn/cuda_gr/src/gpuBSSNExample.cpp:267-299: `#pragma omp parallel for` over
// blocks, one bssnrhs per block). Returns the wall-clock seconds of the loop.
double ref_bssnrhs_blocks_omp(double** rhs, const double** u, int nblocks,
                              const unsigned int* offsets, const double* pmins,
                              const double* pmaxs, const unsigned int* szs,
                              const unsigned int* bflags, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < nblocks; ++b) {
    const unsigned int off = offsets[b];
    const unsigned int bf = bflags[b];
    bssnrhs(rhs, u, off, pmins + 3 * b, pmaxs + 3 * b, szs + 3 * b, bf);
  }
  return omp_get_wtime() - t0;
}

// Hamiltonian, momentum and Psi4 of one block through the reference's own
// `physical_constraints`: con[0..5] = ham, mom0, mom1, mom2, psi4_real, psi4_img
// (bssn/include/grDef.h:40), written at the interior points. Note the reference
// evaluates every stencil with hx in all three directions (physcon.cpp:188-340).
void ref_physical_constraints(double** con, const double** u, unsigned int offset,
                              const double* pmin, const double* pmax, const unsigned int* sz,
                              unsigned int bflag) {
  physical_constraints(con, u, offset, pmin, pmax, sz, bflag);
}

// The reference's 4th-order upwind advective derivatives (bssn/src/derivs.cpp:495-900,
// declared at bssn/include/derivs.h:23-25), for pinning the oracle's restatement.
void ref_deriv42adv(int axis, double* Du, const double* u, double h, const unsigned int* sz,
                    const double* beta, unsigned int bflag) {
  if (axis == 0) deriv42adv_x(Du, u, h, sz, beta, bflag);
  else if (axis == 1) deriv42adv_y(Du, u, h, sz, beta, bflag);
  else deriv42adv_z(Du, u, h, sz, beta, bflag);
}

int ref_max_threads(void) { return omp_get_max_threads(); }

// The reference's analytic test data (bssn/src/grUtils.cpp:15-58).
void ref_fake_initial_data(double x, double y, double z, double* u) {
  bssn::fake_initial_data(x, y, z, u);
}

}  // extern "C"
