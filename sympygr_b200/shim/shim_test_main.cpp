// Test driver for the shim: stands in for the host code (it defines the bssn::
// globals, as the host's parameters.cpp would), fills one block from a raw input
// file, calls bssnrhs (or, with an 8th argument "sep", bssnrhs_sep; "con",
// physical_constraints; "threads", bssnrhs from 4 host threads at once, 3 calls each
// into their own arrays, as the reference's OpenMP block loop calls it) with the
// reference's signature, and writes the 24 RHS (or 6 constraint) arrays.  In the
// threads mode every call's result must equal the first bit for bit (exit code 6
// otherwise).
//   shim_test <in.bin> <out.bin> <n> <pmin> <h> <bflag> <sigma> [sep|con|threads]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

void bssnrhs(double** uzipVarsRHS, const double** uZipVars, const unsigned int& offset,
             const double* ptmin, const double* ptmax, const unsigned int* sz,
             const unsigned int& bflag);
void physical_constraints(double** uZipConVars, const double** uZipVars, const unsigned int& offset,
                          const double* pmin, const double* pmax, const unsigned int* sz,
                          const unsigned int& bflag);
void bssnrhs_sep(double** uzipVarsRHS, const double** uZipVars, const unsigned int& offset,
                 const double* ptmin, const double* ptmax, const unsigned int* sz,
                 const unsigned int& bflag);

namespace bssn {
unsigned int BSSN_LAMBDA[4] = {1, 1, 1, 1};
double BSSN_LAMBDA_F[2] = {1.0, 0.0};
double ETA_CONST = 2.0;
double ETA_R0 = 50.0;
double ETA_DAMPING_EXP = 1.0;
double KO_DISS_SIGMA = 0.01;
}  // namespace bssn

int main(int argc, char** argv) {
  if (argc != 8 && argc != 9) return 2;
  const bool con = argc == 9 && argv[8][0] == 'c';
  const bool sep = argc == 9 && argv[8][0] == 's';
  const bool threads = argc == 9 && argv[8][0] == 't';
  const unsigned n = (unsigned)std::atoi(argv[3]);
  const double p0 = std::atof(argv[4]), h = std::atof(argv[5]);
  const unsigned bflag = (unsigned)std::atoi(argv[6]);
  bssn::KO_DISS_SIGMA = std::atof(argv[7]);
  const size_t npad = (size_t)n * n * n;
  const int nout = con ? 6 : 24;
  std::vector<double> u(24 * npad), r(nout * npad, 0.0);
  FILE* f = std::fopen(argv[1], "rb");
  if (!f || std::fread(u.data(), sizeof(double), u.size(), f) != u.size()) return 3;
  std::fclose(f);
  const double* up[24];
  double* rp[24];
  for (int v = 0; v < 24; ++v) {
    up[v] = u.data() + v * npad;
    rp[v] = v < nout ? r.data() + v * npad : nullptr;
  }
  const double pmin[3] = {p0, p0, p0}, pmax[3] = {p0 + (n - 1) * h, p0 + (n - 1) * h, p0 + (n - 1) * h};
  const unsigned sz[3] = {n, n, n};
  const unsigned offset = 0;
  try {
    if (con)
      physical_constraints(rp, up, offset, pmin, pmax, sz, bflag);
    else if (sep)
      bssnrhs_sep(rp, up, offset, pmin, pmax, sz, bflag);
    else
      bssnrhs(rp, up, offset, pmin, pmax, sz, bflag);
  } catch (...) {
    return 4;
  }
  if (threads) {
    constexpr int kThreads = 4, kCalls = 3;
    std::vector<std::vector<double>> outs(kThreads, std::vector<double>(24 * npad, 0.0));
    std::vector<int> bad(kThreads, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < kThreads; ++t)
      pool.emplace_back([&, t]() {
        double* tp[24];
        for (int v = 0; v < 24; ++v) tp[v] = outs[t].data() + v * npad;
        for (int c = 0; c < kCalls; ++c) {
          try {
            bssnrhs(tp, up, offset, pmin, pmax, sz, bflag);
          } catch (...) {
            bad[t] = 1;
            return;
          }
          if (std::memcmp(outs[t].data(), r.data(), r.size() * sizeof(double)) != 0) bad[t] = 1;
        }
      });
    for (std::thread& th : pool) th.join();
    for (int t = 0; t < kThreads; ++t)
      if (bad[t]) return 6;
  }
  f = std::fopen(argv[2], "wb");
  if (!f || std::fwrite(r.data(), sizeof(double), r.size(), f) != r.size()) return 5;
  std::fclose(f);
  return 0;
}
