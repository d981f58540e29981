/* Driver for the sanitizer check of the oracle: one block through the oracle's right-hand
 * side (standard and upwind mode), its derivative slots and its constraints, built with
 * -fsanitize=address,undefined.  Fills the block with smooth data of its own so it needs
 * nothing else; prints a checksum. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "bssn_oracle.h"

int main(void) {
  const unsigned sz[3] = {14, 13, 16};
  const unsigned flags[4] = {0x00, 0x3F, 0x15, 0x2A};
  const long npad = (long)sz[0] * sz[1] * sz[2];
  const unsigned offset = 7;
  double *u[24], *r[24], *c[4];
  for (int v = 0; v < 24; ++v) {
    u[v] = (double *)malloc(sizeof(double) * (offset + npad));
    r[v] = (double *)calloc(offset + npad, sizeof(double));
    for (long p = 0; p < offset + npad; ++p)
      u[v][p] = 0.3 * sin(0.37 * p + 1.3 * v) + ((v == 0 || v == 1 || v == 12 || v == 15 || v == 17) ? 1.0 : 0.0);
  }
  for (int k = 0; k < 4; ++k) c[k] = (double *)calloc(offset + npad, sizeof(double));
  const double pmin[3] = {-0.4, 0.1, -0.2}, pmax[3] = {0.25, 0.7, 0.5};
  bssn_oracle_params prm = {{1, 1, 1, 1}, {1.0, 0.0}, 2.0, 0.3, 2.0, 0.2};
  const long ni = (long)(sz[0] - 6) * (sz[1] - 6) * (sz[2] - 6);
  double *slots = (double *)malloc(sizeof(double) * BSSN_ORACLE_NUM_SLOTS * ni);
  double sum = 0.0;
  for (int f = 0; f < 4; ++f) {
    bssn_oracle_rhs(r, (const double *const *)u, offset, pmin, pmax, sz, flags[f], &prm);
    for (int v = 0; v < 24; ++v) sum += r[v][offset + npad / 2];
    bssn_oracle_rhs_adv(r, (const double *const *)u, offset, pmin, pmax, sz, flags[f], &prm);
    for (int v = 0; v < 24; ++v) sum += r[v][offset + npad / 2];
    bssn_oracle_derivative_slots(slots, (const double *const *)u, offset, pmin, pmax, sz, flags[f]);
    sum += slots[ni / 2];
    bssn_oracle_block_constraints(c, (const double *const *)u, offset, pmin, pmax, sz, flags[f]);
    sum += c[0][offset + npad / 2];
  }
  printf("checksum %.17g\n", sum);
  for (int v = 0; v < 24; ++v) {
    free(u[v]);
    free(r[v]);
  }
  for (int k = 0; k < 4; ++k) free(c[k]);
  free(slots);
  return isfinite(sum) ? 0 : 1;
}
