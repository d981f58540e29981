// TEST INFRASTRUCTURE ONLY -- declarations that let the reference's generated
// constraint evaluator bssn/CodeGen/physcon.cpp compile unmodified.
//
// physcon.cpp includes "physcon.h" and "gr.h", neither of which the reference tree
// ships. It also differentiates every constraint input twice but allocates second
// derivatives only for gt0..gt5 and chi (physcon.cpp:62-161 against :166-340): the
// writes into grad2_*_{Gt0,Gt1,Gt2,K,At0..At5} name arrays that it never declares and
// never reads. This header declares those names as null pointers at file scope and
// routes the stencil calls through wrappers that skip a null destination, so the
// file compiles as written and computes exactly what it would with the arrays
// present.
#ifndef ORACLE_REF_SHIM_PHYSCON_H
#define ORACLE_REF_SHIM_PHYSCON_H

#include <cmath>
#include <cstdlib>

#include "grDef.h"

void deriv64_x(double *const Dxu, const double *const u, const double dx, const unsigned int *sz, unsigned bflag);
void deriv64_y(double *const Dyu, const double *const u, const double dy, const unsigned int *sz, unsigned bflag);
void deriv64_z(double *const Dzu, const double *const u, const double dz, const unsigned int *sz, unsigned bflag);
void deriv64_xx(double *const Du, const double *const u, const double dx, const unsigned int *sz, unsigned bflag);
void deriv64_yy(double *const Du, const double *const u, const double dy, const unsigned int *sz, unsigned bflag);
void deriv64_zz(double *const Du, const double *const u, const double dz, const unsigned int *sz, unsigned bflag);

namespace physcon_shim {
// deriv_x -> deriv64_x and so on: the 6th-order build (bssn/include/derivs.h:87-100)
inline void x(double *out, const double *in, double h, const unsigned int *sz, unsigned int f) { if (out) ::deriv64_x(out, in, h, sz, f); }
inline void y(double *out, const double *in, double h, const unsigned int *sz, unsigned int f) { if (out) ::deriv64_y(out, in, h, sz, f); }
inline void z(double *out, const double *in, double h, const unsigned int *sz, unsigned int f) { if (out) ::deriv64_z(out, in, h, sz, f); }
inline void xx(double *out, const double *in, double h, const unsigned int *sz, unsigned int f) { if (out) ::deriv64_xx(out, in, h, sz, f); }
inline void yy(double *out, const double *in, double h, const unsigned int *sz, unsigned int f) { if (out) ::deriv64_yy(out, in, h, sz, f); }
inline void zz(double *out, const double *in, double h, const unsigned int *sz, unsigned int f) { if (out) ::deriv64_zz(out, in, h, sz, f); }
}  // namespace physcon_shim

#define deriv_x physcon_shim::x
#define deriv_y physcon_shim::y
#define deriv_z physcon_shim::z
#define deriv_xx physcon_shim::xx
#define deriv_yy physcon_shim::yy
#define deriv_zz physcon_shim::zz

// second derivatives physcon.cpp writes but never allocates or reads
#define PHYSCON_SHIM_UNUSED(v)                                                          \
  static double *const grad2_0_0_##v = nullptr, *const grad2_0_1_##v = nullptr,          \
                       *const grad2_0_2_##v = nullptr, *const grad2_1_1_##v = nullptr,   \
                       *const grad2_1_2_##v = nullptr, *const grad2_2_2_##v = nullptr;
PHYSCON_SHIM_UNUSED(Gt0)
PHYSCON_SHIM_UNUSED(Gt1)
PHYSCON_SHIM_UNUSED(Gt2)
PHYSCON_SHIM_UNUSED(K)
PHYSCON_SHIM_UNUSED(At0)
PHYSCON_SHIM_UNUSED(At1)
PHYSCON_SHIM_UNUSED(At2)
PHYSCON_SHIM_UNUSED(At3)
PHYSCON_SHIM_UNUSED(At4)
PHYSCON_SHIM_UNUSED(At5)
#undef PHYSCON_SHIM_UNUSED

// the reference's entry point (physcon.cpp:12-15)
void physical_constraints(double **uZipConVars, const double **uZipVars, const unsigned int &offset,
                          const double *pmin, const double *pmax, const unsigned int *sz,
                          const unsigned int &bflag);

#endif
