/*
 * CPU oracle: MUSCL / NND2 / first-order primitive reconstruction with the
 * Roe, AUSM+ and HLLC Riemann solvers (src/InviscidScheme.cu,
 * src/Reconstruction.cu, src/Limiter.cuh).  TEST INFRASTRUCTURE ONLY.
 */
#include "oracle.h"

#include <stdio.h>
#include <stdlib.h>

void orc_roe_like_inviscid(orc_zone *z, const orc_param *p) {
  (void)z; (void)p;
  fprintf(stderr, "oracle: MUSCL Riemann-solver schemes are not restated in this build\n");
  abort();
}
