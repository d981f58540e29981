// Host build of the generated device algebra (sympygr_b200/csrc/generated/
// bssn_rhs_algebra.cuh; with a second argument "con" the constraint algebra
// bssn_constraints_algebra.cuh; "adv" the upwind-mode algebra bssn_rhs_algebra_adv.cuh;
// "advsame" the oracle's upwind-mode algebra fed its advective slots from the centred
// first derivatives, against the oracle's standard algebra; "split" the two-part
// algebra bssn_rhs_algebra_split.cuh, both parts in turn) next to the oracle's C
// functions, at seeded random points. Prints the largest norm-wise relative difference
// per output over all points.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#define __device__
#define __forceinline__ inline
using std::sqrt;
#include <cstring>
#include "bssn_constraints_algebra.cuh"
#include "bssn_rhs_algebra.cuh"
#include "bssn_rhs_algebra_adv.cuh"
#include "bssn_rhs_algebra_split.cuh"
extern "C" void bssn_oracle_algebra(const double*, const double*, const double*, double, double*);
extern "C" void bssn_oracle_constraints(const double*, const double*, double*);
extern "C" void bssn_oracle_algebra_adv(const double*, const double*, const double*, double, double*);
struct In {
  const double* u_;
  const double* d_;
  double u(int v) const { return u_[v]; }
  double d(int s) const { return d_[s]; }
};
struct Sink {
  double* o;
  void put(int v, double x) { o[v] = x; }
};
int main(int argc, char** argv) {
  const int npts = argc > 1 ? std::atoi(argv[1]) : 2000;
  const bool con = argc > 2 && std::strcmp(argv[2], "con") == 0;
  const bool adv = argc > 2 && std::strcmp(argv[2], "adv") == 0;
  const bool advsame = argc > 2 && std::strcmp(argv[2], "advsame") == 0;
  const bool split = argc > 2 && std::strcmp(argv[2], "split") == 0;
  const int nout = con ? 4 : 24;
  std::mt19937_64 g(12345);
  std::uniform_real_distribution<double> U(-0.3, 0.3);
  double maxdiff[24] = {0}, maxref[24] = {0};
  const double par[6] = {1, 1, 1, 1, 1, 0};
  const b200bssn::AlgebraParams<double> prm{1, 1, 1, 1, 1, 0};
  for (int t = 0; t < npts; ++t) {
    double u[24], d[210], a[24], b[24];
    for (double& x : u) x = U(g);
    u[0] = 0.8 + U(g);
    u[1] = 0.8 + U(g);
    u[12] = 1 + 0.3 * U(g);
    u[15] = 1 + 0.3 * U(g);
    u[17] = 1 + 0.3 * U(g);
    for (double& x : d) x = U(g);
    const double eta = 2.0 + U(g);
    In in{u, d};
    Sink s{a};
    if (con) {
      b200bssn::bssn_constraints_algebra<double>(in, s);
      bssn_oracle_constraints(u, d, b);
    } else if (adv) {
      b200bssn::bssn_rhs_algebra_adv<double>(in, s, prm, eta);
      bssn_oracle_algebra_adv(u, d, par, eta, b);
    } else if (split) {
      for (double& x : a) x = NAN;  // every output must be written by exactly one part
      b200bssn::RhsAlgebraPart<0>::run<double>(in, s, prm, eta);
      b200bssn::RhsAlgebraPart<1>::run<double>(in, s, prm, eta);
      bssn_oracle_algebra(u, d, par, eta, b);
    } else if (advsame) {
      for (int k = 0; k < 72; ++k) d[138 + k] = d[k];  // agrad_a_<v> = grad_a_<v>
      bssn_oracle_algebra_adv(u, d, par, eta, a);
      bssn_oracle_algebra(u, d, par, eta, b);
    } else {
      b200bssn::bssn_rhs_algebra<double>(in, s, prm, eta);
      bssn_oracle_algebra(u, d, par, eta, b);
    }
    for (int v = 0; v < nout; ++v) {
      const double dv = std::fabs(a[v] - b[v]);
      maxdiff[v] = std::isnan(dv) ? INFINITY : std::fmax(maxdiff[v], dv);  // NaN: unwritten
      maxref[v] = std::fmax(maxref[v], std::fabs(b[v]));
    }
  }
  for (int v = 0; v < nout; ++v) std::printf("%d %.6e\n", v, maxdiff[v] / std::fmax(maxref[v], 1e-300));
  return 0;
}
