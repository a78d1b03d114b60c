/*
 * CPU oracle for the COREFL per-stage right-hand side and update.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C (C99 + OpenMP) restatement of
 * the reference solver's FP64 routines, written to follow the reference's
 * arithmetic order so that the CUDA path can be checked against it.  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may load
 * it; the product library never links or calls it.
 *
 * Layout: every field is a ghost-padded, column-major structure of arrays in
 * the reference's ggxl::VectorField3D form (src/gxl_lib/Array.cuh:246-322):
 *   A(i,j,k,l) = a[(k+g)*(my+2g)*(mx+2g) + (j+g)*(mx+2g) + (i+g) + l*sz]
 * with sz = (mx+2g)(my+2g)(mz+2g) and g the array's ghost width.
 */
#ifndef COREFL_ORACLE_H
#define COREFL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_SPEC 20
#define ORC_MAX_REAC 64

/* Boundary face description (reference src/Mesh.cpp:14-31 register_boundary):
 * face 0/1/2 = i/j/k, direction -1 (min side) or +1 (max side),
 * label 6 = outflow, 8 = periodic, 3 = symmetry, 2 = no-slip wall, 5 = inflow. */
typedef struct {
  int face, direction, label;
} orc_face;

typedef struct {
  int mx, my, mz, ngg;
  /* arrays with ngg ghosts */
  double *cv, *bv, *sv, *qn, *metric, *jac, *mul, *mach;
  double *fFlux, *gFlux, *hFlux;
  /* mixture-only arrays with ngg ghosts */
  double *acoustic_speed, *gamma, *thermal_conductivity, *rho_D, *reaction_timeScale;
  /* 0 ghosts */
  double *dq, *dt_local, *Cn;
  /* 1 ghost */
  double *vis_flux;
  /* ngg ghosts, zero outside the interior (hybrid WENO only; may be NULL) */
  double *shock_sensor;
  /* the step's dt as DParameter::dt holds it after update_dt_global
   * (src/DParameter.cu:396-398); read by the positive-preserving limiter */
  double dt_step;
  /* node y coordinate with ngg ghosts (the mixing-layer inflow; may be NULL) */
  double *y;
  /* applications of a fluctuating inflow so far */
  unsigned long long inflow_draws;
} orc_zone;

/* Species / mechanism tables (reference src/DParameter.cuh:84-130). */
typedef struct {
  int n_spec, n_reac;
  double mw[ORC_MAX_SPEC], imw[ORC_MAX_SPEC], gas_const[ORC_MAX_SPEC];
  /* NASA-7 two-range polynomials, Combustion2Part branch (src/Thermo.cu:385-633) */
  double t_low[ORC_MAX_SPEC], t_mid[ORC_MAX_SPEC], t_high[ORC_MAX_SPEC];
  double low_coeff[ORC_MAX_SPEC][7], high_coeff[ORC_MAX_SPEC][7];
  /* transport (src/Transport.cu:43-165) */
  double geometry[ORC_MAX_SPEC], LJ_potent_inv[ORC_MAX_SPEC], vis_coeff[ORC_MAX_SPEC];
  double WjDivWi_to_One4th[ORC_MAX_SPEC][ORC_MAX_SPEC];
  double sqrt_WiDivWjPl1Mul8[ORC_MAX_SPEC][ORC_MAX_SPEC];
  double binary_diffusivity_coeff[ORC_MAX_SPEC][ORC_MAX_SPEC];
  double kb_over_eps_jk[ORC_MAX_SPEC][ORC_MAX_SPEC];
  double ZRotF298[ORC_MAX_SPEC];
  /* kinetics (src/FiniteRateChem.cu:1466-1605) */
  int reac_type[ORC_MAX_REAC], rev_type[ORC_MAX_REAC];
  int stoi_f[ORC_MAX_REAC][ORC_MAX_SPEC], stoi_b[ORC_MAX_REAC][ORC_MAX_SPEC];
  int reac_order[ORC_MAX_REAC];
  double A[ORC_MAX_REAC], b[ORC_MAX_REAC], Ea[ORC_MAX_REAC];
  double A2[ORC_MAX_REAC], b2[ORC_MAX_REAC], Ea2[ORC_MAX_REAC];
  double third_body_coeff[ORC_MAX_REAC][ORC_MAX_SPEC];
  double troe_alpha[ORC_MAX_REAC], troe_t3[ORC_MAX_REAC], troe_t1[ORC_MAX_REAC], troe_t2[ORC_MAX_REAC];
} orc_mech;

typedef struct {
  int dim, n_var, n_spec, n_scalar, n_reac;
  int inviscid_scheme;   /* 2 Roe, 3 AUSM+, 4 HLLC, 51/52/71/72 WENO */
  int reconstruction;    /* 1 first order, 2 MUSCL, 3 NND2 */
  int limiter;           /* 0 minmod, 1 van Leer */
  int viscous_order;     /* 0 inviscid, 2 second order */
  int positive_preserving;
  int gradPInDiffusionFlux;
  double entropy_fix_factor;
  double Pr, Sc, cfl, dt;
  int fixed_dt;
  double weno_eps_scale, v_ref, rho_ref;
  double sensor_threshold;
  int chem_advance_method;
  int n_face;
  orc_face faces[6];
  const orc_mech *mech;  /* NULL for the calorically perfect air model */
  int shock_sensor;      /* 0 modified Ducros, 1 modified Jameson, 2 density/pressure jump */
  double sensor_eps;     /* shockSensor_epsilon */
  /* the wall of the faces labelled 2 (src/BoundCond.h:88-125): thermal type
   * 0 isothermal at wall_temperature, 1 adiabatic; catalytic type (mixtures)
   * 0 non-catalytic, 1 fully catalytic with mass fractions wall_yk */
  int wall_thermal_type, wall_catalytic_type;
  double wall_temperature;
  double wall_yk[ORC_MAX_SPEC];
  /* the constant inflow of the faces labelled 5 (src/BoundCond.h:22-87):
   * state as Inflow::Inflow derives it, inflow_sub as inflow_subsonic */
  int inflow_subsonic;
  double inflow_density, inflow_u, inflow_v, inflow_w, inflow_pressure, inflow_temperature, inflow_mw;
  double inflow_sv[ORC_MAX_SPEC];
  /* inflow_type 2: the mixing-layer inflow (src/BoundCond.cu:2455-2506) with
   * the lower stream below y = 0; inflow_fluctuation_type 1: white noise on
   * the face velocity, seeded SplitMix64 + Box-Muller deviates */
  int inflow_type;
  double inflow_density_lower, inflow_u_lower, inflow_v_lower, inflow_w_lower, inflow_p_lower, inflow_t_lower;
  double inflow_sv_lower[ORC_MAX_SPEC];
  double inflow_delta_omega;
  int inflow_fluctuation_type;
  double inflow_fluctuation_intensity;
  unsigned long long inflow_seed;
  /* outflow faces (src/BoundCond.h:125-134): if_backPressure, backPressure */
  int outflow_back_pressure_on;
  double outflow_back_pressure;
  /* limit_flow after each stage update (src/RK.cuh:163-164,
   * src/StrangSplitting.cu:602-604) with the bounds of rho, u, v, w, p */
  int limit_flow;
  double limit_ll[5], limit_ul[5];
} orc_param;

/* A face shared by two blocks of a multi-block mesh, as InnerFace holds it
 * after register_boundary (src/Mesh.h:33-59, src/Mesh.cpp:39-172). */
typedef struct {
  int range_start[3], range_end[3];
  int face, direction;
  int target_start[3], target_end[3];
  int target_block, target_face, target_direction;
  int src_tar[3], loop_dir[3], target_loop_dir[3];
  int n_point[3];
} orc_inner_face;

/* InnerFace(...) + register_boundary from the inner-interface records: src and
 * tar are {x1, x2, y1, y2, z1, z2} (1-based, sign-coded), target_block 1-based.
 * Returns 0, or -1 for a record it cannot decode. */
int orc_register_inner_face(int dim, int ngg, const int src[6], const int tar[6], int target_block,
                            orc_inner_face *out);
/* inner_communication (src/DataCommunication.cu:36-102) of one face of zone z
 * with the target block tz (may be z itself). */
void orc_inner_communication(orc_zone *z, orc_zone *tz, const orc_param *p, const orc_inner_face *f);

/* limit_flow (src/TimeAdvanceFunc.cuh:117-230; limits src/DParameter.cu:333-357):
 * interior nodes whose density, velocity or pressure is NaN or outside
 * [ll, ul] take the average of the good nodes of their 3x3x3 neighbourhood
 * inside the block (or their own values clamped to [ll, ul] when none is
 * good), T from the state equation, cv recomputed.  Good and bad are judged
 * on the state before the call, so the result does not depend on the order
 * nodes are visited (the reference's single kernel reads neighbours that
 * other threads may be rewriting; the two agree wherever no two bad nodes
 * are neighbours).  Returns the number of nodes repaired. */
int orc_limit_flow(orc_zone *z, const orc_param *p, const double ll[5], const double ul[5]);
/* halo of a block face shared with another rank's block (src/DataCommunication.cu:210-307) */
long orc_halo_size(const orc_zone *z, const orc_param *p, int face);
void orc_halo_pack(const orc_zone *z, const orc_param *p, int face, int direction, double *buf);
void orc_halo_assign(orc_zone *z, const orc_param *p, int face, int direction, const double *buf);
/* uniform deviate n of face node `node` at inflow application `call` */
double orc_noise_uniform(unsigned long long seed, unsigned long long call, unsigned long long node,
                         unsigned long long n);

/* zone memory management (host, zero-filled) */
int orc_zone_alloc(orc_zone *z, int mx, int my, int mz, int ngg, int n_var, int n_spec, int n_scalar);
void orc_zone_free(orc_zone *z);

/* building blocks (each cites its reference routine in oracle.c) */
void orc_compute_cv_from_bv(orc_zone *z, const orc_param *p);
void orc_update_physical_properties(orc_zone *z, const orc_param *p);
void orc_local_time_step(orc_zone *z, const orc_param *p);
double orc_global_time_step(const orc_zone *z);
void orc_compute_inviscid_flux(orc_zone *z, const orc_param *p);
void orc_compute_viscous_flux(orc_zone *z, const orc_param *p);
void orc_update_cv_and_bv_rk(orc_zone *z, const orc_param *p, double dt, int rk);
void orc_apply_boundary_conditions(orc_zone *z, const orc_param *p);
void orc_eliminate_k_gradient(orc_zone *z, const orc_param *p);
/* compute_shock_sensor (src/FieldOperation.cu:74-179) on the interior nodes */
void orc_compute_shock_sensor(orc_zone *z, const orc_param *p);
/* One SSP-RK3 step (reference src/RK.cuh:84-212); returns the dt used. */
double orc_rk3_step(orc_zone *z, const orc_param *p, double dt_fixed);
/* Stage update with dq - Cn (reference src/StrangSplitting.cu:504-562). */
void orc_update_cv_and_bv_rk_wu(orc_zone *z, const orc_param *p, double dt, int rk);
void orc_local_time_step_without_reaction(orc_zone *z, const orc_param *p);
/* One step of Wu's splitting (reference src/StrangSplitting.cu:683-861); returns the dt used. */
double orc_wu_splitting_step(orc_zone *z, const orc_param *p, double dt_fixed);

/* scalar WENO reconstructions (reference src/WENO.cu:3059-3222) */
double orc_weno5(const double *vp, const double *vm, double eps, int if_shock);
double orc_weno7(const double *vp, const double *vm, double eps, int if_shock);

/* Sutherland viscosity (reference src/Transport.cu:6-9) */
double orc_sutherland(double t);

int orc_num_threads(void);

/* mixture thermo and kinetics (oracle_mix.c) */
void orc_enthalpy_and_cp(const orc_mech *m, double t, double *h, double *cp);
void orc_cp(const orc_mech *m, double t, double *cp);
void orc_gibbs_div_rt(const orc_mech *m, double t, double *g);
void orc_forward_rate(const orc_mech *m, double t, const double *c, double *kf);
void orc_backward_rate(const orc_mech *m, double t, const double *kf, const double *c, double *kb);
void orc_rate_of_progress(const orc_mech *m, const double *kf, const double *kb, const double *c, double *q1,
                          double *q2);
void orc_chemical_source(const orc_mech *m, const double *q1, const double *q2, double *omega_d, double *omega);
void orc_solve_chem_system(double *lhs, double *rhs, int dim);
/* Wu-splitting reaction step over the zone (point implicit when
 * chem_advance_method == 1); nsub_out (N ints, may be NULL) receives the
 * number of substeps taken per node. */
void orc_wu_reaction_step(orc_zone *z, const orc_param *p, double dt, int *nsub_out);
/* explicit finite-rate source into dq and the reaction time scale */
void orc_finite_rate_chemistry(orc_zone *z, const orc_param *p);

#ifdef __cplusplus
}
#endif
#endif
