// Link-compatible replacement for the reference's per-block entry point
//
//   void bssnrhs(double **uzipVarsRHS, const double **uZipVars,
//                const unsigned int &offset, const double *ptmin, const double *ptmax,
//                const unsigned int *sz, const unsigned int &bflag);
//                                           (bssn/include/rhs.h:33-36, bssn/src/rhs.cpp:80)
//
// Compiled into the host code instead of bssn/src/rhs.cpp's bssnrhs, it reads the
// same solver globals (declared below exactly as bssn/include/parameters.h
// declares them; the host's parameters.cpp defines them) and evaluates the block
// on the GPU through the C ABI (b200bssn_rhs).  Each host thread gets its own
// library context, so the reference's OpenMP block loop
// (bssn/cuda_gr/src/gpuBSSNExample.cpp:267-299) keeps working unchanged.
//
// The staged variant bssnrhs_sep (bssn/include/rhs.h:39, bssn/src/rhs.cpp:392-825),
// which bssnRHS calls instead when built with BSSN_RHS_STAGED_COMP, computes the same
// right-hand side one equation group at a time (it agrees with bssnrhs to ~2e-15);
// it is defined here too, on the same GPU path.
//
// It also replaces the reference's constraint evaluator
//
//   void physical_constraints(double **uZipConVars, const double **uZipVars,
//                             const unsigned int &offset, const double *pmin,
//                             const double *pmax, const unsigned int *sz,
//                             const unsigned int &bflag);   (bssn/CodeGen/physcon.cpp:12-15)
//
// writing uZipConVars[C_HAM..C_MOM2] (bssn/include/grDef.h:40) at the interior
// points; the Psi4 arrays (C_PSI4_REAL, C_PSI4_IMG) are left untouched.
//
// Environment: B200BSSN_DEVICE (CUDA device, default 0), B200BSSN_PRECISION
// ("fp64" default, or "mixed").  The reference function returns nothing; a
// failure here throws std::runtime_error with the library's message.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "b200bssn.h"

namespace bssn {
extern unsigned int BSSN_LAMBDA[4];   // bssn/include/parameters.h:221
extern double BSSN_LAMBDA_F[2];       // :224
extern double ETA_CONST;              // :234
extern double ETA_R0;                 // :237
extern double ETA_DAMPING_EXP;        // :243
extern double KO_DISS_SIGMA;          // :252
}  // namespace bssn

namespace {

struct ThreadCtx {
  b200bssn_ctx* ctx = nullptr;
  ~ThreadCtx() {
    if (ctx) b200bssn_destroy(ctx);
  }
};

b200bssn_ctx* thread_ctx() {
  thread_local ThreadCtx tc;
  if (!tc.ctx) {
    const char* d = std::getenv("B200BSSN_DEVICE");
    const int dev = d ? std::atoi(d) : 0;
    const int rc = b200bssn_create(&tc.ctx, dev);
    if (rc != B200BSSN_OK)
      throw std::runtime_error(std::string("bssnrhs: b200bssn_create failed: ") +
                               b200bssn_status_string(rc));
  }
  return tc.ctx;
}

uint32_t precision_from_env() {
  const char* p = std::getenv("B200BSSN_PRECISION");
  return (p && std::strcmp(p, "mixed") == 0) ? B200BSSN_MIXED : B200BSSN_FP64;
}

}  // namespace

void bssnrhs(double** uzipVarsRHS, const double** uZipVars, const unsigned int& offset,
             const double* ptmin, const double* ptmax, const unsigned int* sz,
             const unsigned int& bflag) {
  b200bssn_params p;
  b200bssn_default_params(&p);
  for (int i = 0; i < 4; ++i) p.lambda[i] = bssn::BSSN_LAMBDA[i];
  p.lambda_f[0] = bssn::BSSN_LAMBDA_F[0];
  p.lambda_f[1] = bssn::BSSN_LAMBDA_F[1];
  p.eta_const = bssn::ETA_CONST;
  p.eta_r0 = bssn::ETA_R0;
  p.eta_damping_exp = bssn::ETA_DAMPING_EXP;
  p.ko_sigma = bssn::KO_DISS_SIGMA;
  p.precision = precision_from_env();
  b200bssn_ctx* ctx = thread_ctx();
  const uint32_t usz[3] = {sz[0], sz[1], sz[2]};
  const int rc = b200bssn_rhs(ctx, uzipVarsRHS, uZipVars, offset, ptmin, ptmax, usz, bflag, &p);
  if (rc != B200BSSN_OK)
    throw std::runtime_error(std::string("bssnrhs: ") + b200bssn_status_string(rc) + " (" +
                             b200bssn_last_error(ctx) + ")");
}

void bssnrhs_sep(double** uzipVarsRHS, const double** uZipVars, const unsigned int& offset,
                 const double* ptmin, const double* ptmax, const unsigned int* sz,
                 const unsigned int& bflag) {
  bssnrhs(uzipVarsRHS, uZipVars, offset, ptmin, ptmax, sz, bflag);
}

void physical_constraints(double** uZipConVars, const double** uZipVars, const unsigned int& offset,
                          const double* pmin, const double* pmax, const unsigned int* sz,
                          const unsigned int& bflag) {
  b200bssn_ctx* ctx = thread_ctx();
  const uint32_t usz[3] = {sz[0], sz[1], sz[2]};
  const int rc = b200bssn_physical_constraints(ctx, uZipConVars, uZipVars, offset, pmin, pmax, usz,
                                               bflag, precision_from_env());
  if (rc != B200BSSN_OK)
    throw std::runtime_error(std::string("physical_constraints: ") + b200bssn_status_string(rc) +
                             " (" + b200bssn_last_error(ctx) + ")");
}
