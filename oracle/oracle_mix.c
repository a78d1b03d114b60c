/*
 * CPU oracle, mixture model: thermo, transport, mixture WENO characteristic
 * projection, species viscous terms, MUSCL + Roe/AUSM+/HLLC, finite-rate
 * chemistry.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

static void not_yet(const char *what) {
  fprintf(stderr, "oracle: %s is not available in this build of the oracle\n", what);
  abort();
}

void orc_weno_face_mixture(const orc_zone *z, const orc_param *p, int dir, long idx, double kx, double ky,
                           double kz, double eps_ref, double *fc) {
  (void)z; (void)p; (void)dir; (void)idx; (void)kx; (void)ky; (void)kz; (void)eps_ref; (void)fc;
  not_yet("mixture WENO");
}
void orc_positive_preserving_face(const orc_zone *z, const orc_param *p, int dir, long idx, double *fc) {
  (void)z; (void)p; (void)dir; (void)idx; (void)fc;
  not_yet("positive-preserving limiter");
}
void orc_roe_like_inviscid(orc_zone *z, const orc_param *p) { (void)z; (void)p; not_yet("MUSCL Riemann solvers"); }
void orc_viscous_species_face(const orc_zone *z, const orc_param *p, int dir, int i, int j, int k,
                              const double gm[9], const double gk[3], double *fv) {
  (void)z; (void)p; (void)dir; (void)i; (void)j; (void)k; (void)gm; (void)gk; (void)fv;
  not_yet("species diffusion");
}
void orc_temperature_and_pressure(orc_zone *z, const orc_param *p, long id, double e) {
  (void)z; (void)p; (void)id; (void)e; not_yet("mixture T-Newton");
}
void orc_total_energy_mixture(orc_zone *z, const orc_param *p, long id) { (void)z; (void)p; (void)id; not_yet("mixture energy"); }
void orc_update_physical_properties_mixture_point(orc_zone *z, const orc_param *p, long id) {
  (void)z; (void)p; (void)id; not_yet("mixture properties");
}
double orc_mixture_max_diffuse_vel(const orc_zone *z, const orc_param *p, long id) {
  (void)z; (void)p; (void)id; not_yet("mixture dt"); return 0;
}
