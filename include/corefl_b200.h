/*
 * corefl_b200 — B200 (sm_100a) implementation of the COREFL per-stage
 * right-hand side and SSP-RK3 update, behind a plain C ABI.
 *
 * Every entry point returns 0 on success and a negative cfk_status on error;
 * cfk_last_error() gives the message.  Streams are passed as void* so that a
 * binder needs no CUDA headers (pass a cudaStream_t, or NULL for the legacy
 * default stream).  All arrays are FP64 device pointers in the reference's
 * ggxl::VectorField3D layout (reference src/gxl_lib/Array.cuh:246-322):
 *
 *   A(i,j,k,l) = a[(k+g)*(my+2g)*(mx+2g) + (j+g)*(mx+2g) + (i+g) + l*sz],
 *   sz = (mx+2g)(my+2g)(mz+2g),
 *
 * g = ngg for cv, bv, sv, qn, metric, jac and the property arrays; g = 0 for
 * dq, dt_local and Cn — the widths the reference allocates in
 * Field::setup_device_memory (reference src/Field.cu:422-655).
 */
#ifndef COREFL_B200_H
#define COREFL_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum cfk_status {
  CFK_OK = 0,
  CFK_ERR_ARG = -1,      /* bad argument or unsupported setting */
  CFK_ERR_CUDA = -2,     /* a CUDA call failed */
  CFK_ERR_STATE = -3,    /* call out of order (e.g. no zone bound) */
  CFK_ERR_NUMERIC = -4,  /* a bounded iteration gave up (see cfk_last_error) */
  CFK_ERR_IO = -5        /* file could not be read or parsed */
};

typedef struct cfk_ctx cfk_ctx;

#define CFK_MAX_SPEC 9   /* species of a mechanism (cfk_mechanism, cfk_wall) */
#define CFK_MAX_REAC 24  /* reactions of a mechanism */

/* A boundary face of the block (reference src/Mesh.cpp:14-31, Boundary).
 * face 0/1/2 = i/j/k, direction -1 = min side, +1 = max side;
 * label 6 = outflow, 8 = periodic, 3 = symmetry, 2 = no-slip wall (cfk_param.wall),
 * 5 = inflow (cfk_param.inflow); outflow faces read cfk_param.outflow. */
typedef struct cfk_face {
  int face, direction, label;
} cfk_face;

/* The no-slip wall of the faces labelled 2 (reference src/BoundCond.h:88-125,
 * Wall, as read by src/BoundCond.cpp:480-528).  thermal_type 0 isothermal at
 * `temperature`, 1 adiabatic (the reference's third type, equilibrium
 * radiation, needs the wall-distance field and is rejected).  catalytic_type
 * (mixtures only; ignored for air, as in the reference) 0 non-catalytic —
 * the wall takes its inner neighbour's mass fractions — or 1 fully catalytic
 * with the wall mass fractions yk[0..n_spec). */
typedef struct cfk_wall {
  int thermal_type, catalytic_type;
  double temperature;
  double yk[CFK_MAX_SPEC];
} cfk_wall;

/* A face this block shares with a block of the same mesh: the reference's
 * InnerFace after register_boundary (reference src/Mesh.h:33-59,
 * src/Mesh.cpp:39-172).  0-based node indices; range_* run over this block's
 * face nodes and the ngg ghost layers behind them (face direction) and the
 * face's own nodes (tangential directions, corners excluded); node n of the
 * loop maps to target node target_start[a] + target_loop_dir[a] *
 * d[src_tar[a]] with d[b] = loop_dir[b] * n[b].  Build it with
 * cfk_register_inner_face. */
typedef struct cfk_inner_face {
  int range_start[3], range_end[3];
  int face, direction;               /* normal axis 0/1/2; -1 min side, +1 max side */
  int target_start[3], target_end[3];
  int target_block, target_face, target_direction;
  int src_tar[3], loop_dir[3], target_loop_dir[3];
  int n_point[3];
} cfk_inner_face;

/* The inflow of the faces labelled 5 (reference src/BoundCond.h:22-87,
 * Inflow): the state the reference derives in Inflow::Inflow
 * (src/BoundCond.cpp:9-260) — density, velocity, pressure, temperature, the
 * mean molecular weight (mixtures) and the scalars (mass fractions).
 * subsonic = the reference's inflow_sub: where the normal Mach number at the
 * face is not below -1 the face takes the characteristic combination of the
 * inflow state and the inner node.
 * inflow_type 0: the constant state.  inflow_type 2 (mixing layer, the
 * reference's problem_type 1): u = (u + u_lower)/2 + (u - u_lower)/2 *
 * tanh(2 y / delta_omega), and the other variables and scalars from the
 * upper set (the fields above) where y >= 0, from the *_lower set below
 * (src/BoundCond.cu:2455-2478); needs the zone's y plane.
 * fluctuation_type 1 (white noise, src/BoundCond.cu:2290-2313, 2479-2505,
 * 2573-2596): normal deviates added to the face velocity every time the
 * boundary conditions are applied — inflow_type 2: u, v, w each plus
 * N(0,1) * fluctuation_intensity * u * exp(-y^2); inflow_type 0: u plus
 * N(0,1) * fluctuation_intensity * |V|.  The deviates are this library's own
 * seeded counter-based stream (SplitMix64 hashing of seed, face node and the
 * context's count of applications, Box-Muller), not curand's: runs repeat
 * bit for bit for a given seed.  Not subsonic with inflow_type 2. */
typedef struct cfk_inflow {
  int subsonic;
  double density, u, v, w, pressure, temperature, mw;
  double sv[CFK_MAX_SPEC];
  int inflow_type;                 /* 0 constant, 2 mixing layer */
  double density_lower, u_lower, v_lower, w_lower, p_lower, t_lower;
  double sv_lower[CFK_MAX_SPEC];
  double delta_omega;              /* initial vorticity thickness, m */
  int fluctuation_type;            /* 0 none, 1 white noise */
  double fluctuation_intensity;
  unsigned long long seed;
} cfk_inflow;

/* The outflow of the faces labelled 6 (reference src/BoundCond.h:125-134,
 * Outflow).  back_pressure_on = the reference's if_backPressure: where the
 * face's normal Mach number is below 1 the ghosts carry the characteristic
 * state at back_pressure; otherwise (and without it) they copy the face. */
typedef struct cfk_outflow {
  int back_pressure_on;
  double back_pressure;
} cfk_outflow;

/* Scalar settings of the path: the DParameter fields it reads
 * (reference src/DParameter.cuh:13-207) plus the boundary list. */
typedef struct cfk_param {
  int dim;                 /* 2 or 3 */
  int n_var;               /* 5 + n_scalar */
  int n_spec;              /* 0 for the air model */
  int n_scalar;
  int n_reac;
  int inviscid_scheme;     /* 2 Roe, 3 AUSM+, 4 HLLC (MUSCL/NND2/1st), 51/52/71/72 WENO */
  int reconstruction;      /* 1 first order, 2 MUSCL, 3 NND2 */
  int limiter;             /* 0 minmod, 1 van Leer */
  int viscous_order;       /* 0, 2 or 8 as in the reference; 4: the added 4th-order collocated scheme */
  int positive_preserving;
  int gradPInDiffusionFlux;
  int fixed_dt;
  int chem_advance_method; /* 0 explicit, 1 point implicit */
  int n_face;
  cfk_face faces[6];
  double entropy_fix_factor;
  double Pr, Sc, cfl, dt;
  double weno_eps_scale;   /* (rho_ref * v_ref)^2, reference src/DParameter.cu:25-28 */
  double v_ref, rho_ref;
  double sensor_threshold; /* shockSensor_threshold; <= 1e-10: WENO nonlinear weights everywhere,
                              above: hybrid UD5/UD7 + WENO5/WENO7 (schemes 52/72) */
  int device;              /* CUDA device ordinal the context runs on */
  int shock_sensor;        /* 0 modified Ducros, 1 modified Jameson, 2 density/pressure jump */
  double sensor_eps;       /* shockSensor_epsilon (reference default -1) */
  cfk_wall wall;           /* read for faces labelled 2 */
  cfk_inflow inflow;       /* read for faces labelled 5 */
  cfk_outflow outflow;     /* read for faces labelled 6 */
  int limit_flow;          /* 1: limit_flow after every stage update (reference src/RK.cuh:163-164,
                              src/StrangSplitting.cu:602-604); needs the bounds below */
  double limit_ll[5];      /* lower bounds of rho, u, v, w, p (reference src/DParameter.cu:333-349:
                              1e-6 rho_inf, -1000 v_inf, 1e-6 p_inf) */
  double limit_ul[5];      /* upper bounds (1e3 rho_inf, 1000 v_inf, 1e3 p_inf) */
} cfk_param;

/* Device pointers of one block, field for field the arrays of the reference's
 * DZone (reference src/Field.h:12-130) that this path reads or writes.
 * Pointers a configuration does not use may be NULL. */
typedef struct cfk_zone {
  int mx, my, mz, ngg;
  double *jac, *metric;          /* 1 and 9 planes, ngg ghosts */
  double *cv, *bv, *sv, *qn;     /* n_var, 6, n_scalar, n_var planes, ngg ghosts */
  double *mul, *mach;            /* ngg ghosts */
  double *acoustic_speed, *gamma, *thermal_conductivity, *rho_D, *reaction_timeScale; /* mixture */
  double *dq, *dt_local, *Cn;    /* n_var, 1, n_var planes, 0 ghosts */
  double *shock_sensor;          /* 1 plane, ngg ghosts, zero-initialised; hybrid schemes only.  NULL: the
                                    context allocates its own */
  double *y;                     /* 1 plane, ngg ghosts: node y coordinate (DZone::y); required by the
                                    mixing-layer inflow and its white noise, else may be NULL */
} cfk_zone;

/* Species, thermo, transport and kinetics tables of a mechanism — the
 * DParameter tables (reference src/DParameter.cuh:84-130) that the mixture
 * and chemistry kernels read.  Up to CFK_MAX_SPEC species and CFK_MAX_REAC
 * reactions; matrices are row-major [reaction][species] or [species][species].
 * reac_type: 0 irreversible, 1 elementary, 3 merged duplicate, 4 third body,
 * 5 Lindemann, 6/7 Troe with 3/4 parameters; rev_type 1 = explicit reverse
 * Arrhenius (REV).  Ea and Ea2 are in K (already divided by R_c). */
typedef struct cfk_mechanism {
  int n_spec, n_reac;
  double mw[CFK_MAX_SPEC];
  double t_low[CFK_MAX_SPEC], t_mid[CFK_MAX_SPEC], t_high[CFK_MAX_SPEC];
  double low[CFK_MAX_SPEC][7], high[CFK_MAX_SPEC][7];
  int geometry[CFK_MAX_SPEC];
  double LJ_potent_inv[CFK_MAX_SPEC], vis_coeff[CFK_MAX_SPEC], ZRotF298[CFK_MAX_SPEC];
  double WjDivWi_to_One4th[CFK_MAX_SPEC][CFK_MAX_SPEC];
  double sqrt_WiDivWjPl1Mul8[CFK_MAX_SPEC][CFK_MAX_SPEC];
  double binary_diffusivity_coeff[CFK_MAX_SPEC][CFK_MAX_SPEC];
  double kb_over_eps_jk[CFK_MAX_SPEC][CFK_MAX_SPEC];
  int reac_type[CFK_MAX_REAC], rev_type[CFK_MAX_REAC], order[CFK_MAX_REAC];
  int stoi_f[CFK_MAX_REAC][CFK_MAX_SPEC], stoi_b[CFK_MAX_REAC][CFK_MAX_SPEC];
  double A[CFK_MAX_REAC], b[CFK_MAX_REAC], Ea[CFK_MAX_REAC];
  double A2[CFK_MAX_REAC], b2[CFK_MAX_REAC], Ea2[CFK_MAX_REAC];
  double third_body_coeff[CFK_MAX_REAC][CFK_MAX_SPEC];
  double troe_alpha[CFK_MAX_REAC], troe_t3[CFK_MAX_REAC], troe_t1[CFK_MAX_REAC], troe_t2[CFK_MAX_REAC];
} cfk_mechanism;

/* ---- context ---------------------------------------------------------- */
int cfk_create(const cfk_param *param, cfk_ctx **out);
int cfk_destroy(cfk_ctx *ctx);
const char *cfk_last_error(const cfk_ctx *ctx);
/* Fill a cfk_param from a reference setup.txt (reference src/Parameter.cpp:38-184,
 * defaults :342-523, derived values :186-340).  Returns CFK_ERR_IO on failure. */
int cfk_param_from_setup(const char *setup_path, cfk_param *out, char *err, size_t err_len);

/* Adopt caller-owned device arrays in place, no copies (the reference's
 * Field::d_ptr / h_ptr arrays). */
int cfk_bind_zone(cfk_ctx *ctx, const cfk_zone *zone);
/* Allocate a zone owned by the context (zero-filled) and bind it; its device
 * pointers are returned in *zone_out. */
int cfk_alloc_zone(cfk_ctx *ctx, int mx, int my, int mz, cfk_zone *zone_out);

/* ---- per-stage entry points (each replaces the reference call named) ---- */
/* dq += viscous flux differences.  Replaces compute_viscous_flux<M>
 * (reference src/ViscousScheme.cu:7-73). */
int cfk_compute_viscous_flux(cfk_ctx *ctx, void *stream);
/* dq -= inviscid flux differences, all directions.  Replaces
 * compute_inviscid_flux<M> (reference src/InviscidScheme.cu:12-26), including
 * compute_convective_term_weno (reference src/WENO.cu:2914-2946). */
int cfk_compute_inviscid_flux(cfk_ctx *ctx, void *stream);
/* Shock sensor of the hybrid schemes on the interior nodes (ghost layers
 * keep 0).  Replaces compute_shock_sensor (reference
 * src/FieldOperation.cu:158-179), called once per step (reference
 * src/RK.cuh:112-117, src/StrangSplitting.cu:19-24); cfk_rk3_step and
 * cfk_wu_splitting_step call it themselves.  No-op unless
 * sensor_threshold > 1e-10. */
int cfk_compute_shock_sensor(cfk_ctx *ctx, void *stream);

/* ---- tile autotuner (no reference counterpart) ---- */
/* The WENO flux kernels come in CFK_TILE_VARIANTS tile shapes per sweep
 * (nodes per column x columns per CTA: x 63x4, 15x16, 31x8; y/z 15x32, 31x16,
 * 63x8 for air and, for mixtures, x 63x4, 127x2, 31x8; y/z 15x16, 31x8, 63x4).
 * A new context starts on variants {2, 1, 1} for air (x 31x8, y/z 31x16: the
 * tuner's choice on large 3-D blocks) and {0, 0, 0} for mixtures, with the
 * viscous form 2 below.  cfk_autotune_tiles times each variant of each sweep on the bound zone (reps launches after one
 * warm-up, into scratch memory: the zone's arrays are not changed), keeps the
 * fastest per direction for all later calls, and reports
 * ms_out[dir * CFK_TILE_VARIANTS + var] (average ms per launch) and
 * choice_out[3]; either may be NULL.  It allocates, so call it outside stream
 * capture.  A no-op for the primitive-variable schemes (one tile shape). */
#define CFK_TILE_VARIANTS 3
int cfk_autotune_tiles(cfk_ctx *ctx, int reps, double *ms_out, int *choice_out, void *stream);
/* For air with viscous_order 2, cfk_autotune_tiles also times the forms of
 * the fused viscous kernel — 0: all per-node inputs staged in shared memory
 * (two plane slots); 1: only u, v, w, T, mu staged, in a three-slot ring
 * filled by cp.async ahead of use, with the metric read through L1, two CTAs
 * per SM; 2: the same with the metric and J of the plane two ahead
 * prefetched into L2 — and keeps the fastest (the same arithmetic; they agree
 * to the last bits).
 * cfk_viscous_variant reads (set = 0) or sets (set = 1) the form in *var;
 * ms (optional, 3 doubles) receives the last autotune's times per launch. */
int cfk_viscous_variant(cfk_ctx *ctx, int set, int *var, double *ms);
/* Sets the tile variant of each sweep (var[3], each 0..CFK_TILE_VARIANTS-1). */
int cfk_set_tile_variants(cfk_ctx *ctx, const int *var);
/* SSP-RK3 stage update of cv and bv/sv.  Replaces update_cv_and_bv_rk<M>
 * (reference src/RK.cuh:224-281). */
int cfk_update_cv_and_bv_rk(cfk_ctx *ctx, double dt, int rk, void *stream);
/* Replaces limit_flow<M> (reference src/TimeAdvanceFunc.cuh:117-220), with the
 * bounds param->limit_ll / limit_ul: every interior node whose density,
 * velocity or pressure is NaN or outside the bounds takes the mean of the
 * in-bounds nodes of its 3x3x3 neighbourhood (clamped to the bounds when there
 * is none), its temperature from the state equation and its cv from bv.  All
 * decisions are taken on the values before the call (the reference reads
 * neighbours while other threads rewrite them).  *n_repaired (may be NULL)
 * receives the number of repaired nodes; it synchronises the stream.  The
 * first call on a context whose param has limit_flow = 0 allocates one byte
 * per node; RK3 and Wu steps call it after each stage update when
 * limit_flow = 1. */
int cfk_limit_flow(cfk_ctx *ctx, long long *n_repaired, void *stream);
/* Halo of a block face shared with a block on another rank: the reference's
 * parallel faces (src/Mesh.cpp:964-995, parallel_communication
 * src/DataCommunication.cu:105-208).  face 0/1/2 and direction -1 (min
 * side) / +1 (max side) name a whole block face over the block's own
 * tangential nodes.  cfk_halo_pack replaces setup_data_to_be_sent (:270-307):
 * it writes, per face node (first tangential axis fastest), the face node and
 * the ngg nodes inside it, each as the 6 basic variables and the n_scalar
 * scalars, into the device buffer buf of cfk_halo_size doubles.
 * cfk_halo_assign replaces assign_data_received (:210-266): from the
 * neighbour's packed buffer it averages the shared face nodes (copies theirs
 * where ours has |V| > 1e-15 and theirs not; leaves ours where ours is at
 * rest), fills the ngg ghost layers from the neighbour's inner layers and
 * sets cv from bv there.  Moving the buffers between ranks is the caller's
 * (NCCL, MPI, a peer copy); the face's own boundary condition is none. */
int cfk_halo_size(cfk_ctx *ctx, int face, long long *n_doubles);
int cfk_halo_pack(cfk_ctx *ctx, int face, int direction, double *buf, void *stream);
int cfk_halo_assign(cfk_ctx *ctx, int face, int direction, const double *buf, void *stream);
/* Replaces update_physical_properties<M> (reference src/FieldOperation.cuh:86-120). */
int cfk_update_physical_properties(cfk_ctx *ctx, void *stream);
/* Replaces compute_cv_from_bv<M> (reference src/FieldOperation.cuh:39-64). */
int cfk_compute_cv_from_bv(cfk_ctx *ctx, void *stream);
/* Replaces DBoundCond::apply_boundary_conditions<M> for outflow, inflow, symmetry,
 * wall and periodic faces (reference src/BoundCond.cu:3489-3619) and, for 2-D blocks,
 * eliminate_k_gradient (reference src/FieldOperation.cu:47-72). */
int cfk_apply_boundary_conditions(cfk_ctx *ctx, void *stream);
/* eliminate_k_gradient on its own (reference src/FieldOperation.cu:47-72): a
 * 2-D block's k = 0 plane copied into its k ghost layers.  The reference calls
 * it after data_communication (reference src/RK.cuh:175-183), so a 2-D
 * multi-block stage calls it again after its cfk_inner_communication calls. */
int cfk_eliminate_k_gradient(cfk_ctx *ctx, void *stream);

/* ---- flowfield files (host only) ------------------------------------------ */
/* One block of a Tecplot V112 binary flowfield file: interior node counts,
 * the ghost width of the host arrays below (the reference's padded layout),
 * and the arrays — coordinates, the 6 basic variables (density, u, v, w,
 * pressure, temperature), n_scalar scalars (species mass fractions) and
 * n_other further planes (Mach number, ...). */
typedef struct cfk_plt_block {
  int mx, my, mz, ngg;
  const double *x, *y, *z;
  const double *bv, *sv, *ov;
} cfk_plt_block;
/* A block to restart: sizes, ghost width and the host arrays to fill. */
typedef struct cfk_plt_target {
  int mx, my, mz, ngg;
  double *bv, *sv;
} cfk_plt_target;
/* Write `path` as the reference's output/flowfield.plt (reference
 * src/FieldIO.h:83-420, FieldIO::write_header + write_common_data_section):
 * one zone per block over its nodes widened by ngg_output ghost layers,
 * variables in the order x, y, z, bv, sv, ov with their min/max pairs, all in
 * double precision.  var_names holds the 9 + n_scalar + n_other names.
 * CFK_ERR_IO if the file cannot be written; err (may be NULL) gets a message. */
int cfk_write_flowfield(const char *path, const cfk_plt_block *blocks, int n_block, int ngg_output,
                        const char *const *var_names, int n_scalar, int n_other, double solution_time,
                        char *err, size_t err_len);
/* Restart from a flowfield file (reference src/Initialize.cu:97-345, the
 * branch where the file's zones are the current blocks in the same order):
 * every variable whose name is a basic variable (density/rho/roe, u, v, w,
 * p/pressure, t/temperature, any case) or one of species_names is read into
 * bv or sv over the file's nodes (the zone may carry up to the block's ngg
 * ghost layers); other variables are skipped.  *solution_time (may be NULL)
 * gets the zones' solution time.  On a truncated file the arrays may be
 * partly filled and CFK_ERR_IO is returned. */
int cfk_read_flowfield(const char *path, const cfk_plt_target *blocks, int n_block,
                       const char *const *species_names, int n_spec, double *solution_time, char *err,
                       size_t err_len);

/* ---- multi-block meshes on one GPU ---------------------------------------- */
/* Build an inner face from the two records of the mesh's inner-interface file
 * (reference src/Mesh.cpp:927-958 and InnerFace::register_boundary,
 * src/Mesh.cpp:39-172): src = this block's 1-based node range
 * {x1, x2, y1, y2, z1, z2}, the normal axis marked by equal ends (1: min side)
 * and, in 3-D, the first tangential axis by negated values; tar = the same
 * for the target block, whose 1-based number is target_block (stored
 * 0-based).  Host-only arithmetic; CFK_ERR_ARG for a record without a normal
 * axis or, in 3-D, without a marked tangential axis. */
int cfk_register_inner_face(int dim, int ngg, const int src[6], const int tar[6], int target_block,
                            cfk_inner_face *out);
/* Read the mesh's inner-interface file (input/boundary_condition/inner%4d.txt,
 * reference src/Mesh.cpp:927-958) and register every face in it: faces[]
 * receives them block by block in file order (at most max_faces), and
 * n_per_block[b] how many belong to block b.  Host only. */
int cfk_read_inner_interface(const char *path, int dim, int ngg, int n_block, cfk_inner_face *faces, int max_faces,
                             int *n_per_block, char *err, size_t err_len);
/* Replaces inner_communication<M> of data_communication for one inner face
 * (reference src/DataCommunication.cu:6-102): this block's ghost nodes behind
 * the face take the target block's primitive variables; on the face itself
 * the two blocks' nodes are averaged, both sides written (a node at rest — a
 * wall — is left alone, and takes the target's values when only the target's
 * node is at rest); this block's cv is recomputed on every node visited.
 * `target` is the neighbouring block's context, or ctx itself; both bound on
 * the same device with the same ngg, dimension and variable counts, and every
 * node the face maps must lie inside both padded blocks (checked on the host,
 * as is a face-normal extent above ngg for both blocks).  Call it per block and
 * per face after every block's cfk_apply_boundary_conditions, in the order
 * the reference visits them. */
int cfk_inner_communication(cfk_ctx *ctx, cfk_ctx *target, const cfk_inner_face *face, void *stream);
/* Local CFL step into dt_local and its minimum.  Replaces local_time_step<M>
 * + global_time_step (reference src/TimeAdvanceFunc.cuh:28-115,
 * src/TimeAdvanceFunc.cu:102-152).  *dt_out is written after a stream sync. */
int cfk_local_time_step(cfk_ctx *ctx, double *dt_out, void *stream);

/* Load the mechanism tables (required when n_spec > 0). */
int cfk_set_mechanism(cfk_ctx *ctx, const cfk_mechanism *mech);
/* Explicit finite-rate source dq[5+l] += J*omega_l and the reaction time
 * scale.  Replaces finite_rate_chemistry (reference src/FiniteRateChem.cu:1388-1464). */
int cfk_finite_rate_chemistry(cfk_ctx *ctx, void *stream);
/* Reaction step of Wu's splitting over dt at every node: n_sub = int(dt/tau)
 * substeps of dt/(n_sub+1) plus the remainder, each an explicit
 * (chem_advance_method 0) or point-implicit (1) 0-D update with the frozen
 * transport term Cn.  Replaces wu_reaction_step (reference
 * src/StrangSplitting.cu:373-421, 43-224).  schedule 0 = one thread per
 * node (the reference's mapping); 1 = persistent work-queue kernel in which
 * each lane pulls the next node when its node is done, so nodes with uneven
 * substep counts do not idle the warp.  Both give identical results.
 * nsub_out (device int[mx*my*mz], may be NULL) receives the substeps per node.
 * n_sub is capped at 100000 per node; CFK_ERR_NUMERIC is reported by the next
 * cfk_stream_sync if a node hit the cap. */
int cfk_wu_reaction_step(cfk_ctx *ctx, double dt, int schedule, int *nsub_out, void *stream);

/* ---- whole steps ------------------------------------------------------ */
/* One SSP-RK3 step: qn <- cv, dt (fixed or CFL), three stages of
 * dq = 0, viscous, inviscid, update, BCs, property update (the loop body of
 * RK3, reference src/RK.cuh:84-212).  When the CFL step is used the dt stays
 * on the device: no host round trip inside the step.  *dt_used (may be NULL)
 * is read back only if non-NULL. */
int cfk_rk3_step(cfk_ctx *ctx, double *dt_used, void *stream);
/* Same step replayed from a CUDA graph captured on first use (the graph is
 * rebuilt if the zone is re-bound). */
int cfk_rk3_step_graph(cfk_ctx *ctx, double *dt_used, void *stream);
/* One step of Wu's splitting for a reacting mixture (the loop body of
 * wu_splitting, reference src/StrangSplitting.cu:683-861): dt fixed or from
 * local_time_step_without_reaction; Cn = viscous + inviscid right-hand side
 * (compute_cn, :15-41); the reaction step over dt with the frozen Cn
 * (schedule 0 one thread per node, 1 work queue), BCs, property update
 * (wu_reaction_subStep, :475-502); SSP-RK3 over dt/2 on dq - Cn with BCs and
 * no property update (wu_RK_subStep, :564-634).  *dt_used (may be NULL)
 * receives the dt; the CFL dt costs one host synchronisation. */
int cfk_wu_splitting_step(cfk_ctx *ctx, int schedule, double *dt_used, void *stream);

/* ---- host <-> device helpers for callers without a CUDA runtime -------- */
int cfk_memcpy_h2d(cfk_ctx *ctx, void *dst_dev, const void *src_host, size_t bytes, void *stream);
int cfk_memcpy_d2h(cfk_ctx *ctx, void *dst_host, const void *src_dev, size_t bytes, void *stream);
/* device to device (snapshot / restore of zone arrays) */
int cfk_memcpy_d2d(cfk_ctx *ctx, void *dst_dev, const void *src_dev, size_t bytes, void *stream);
int cfk_stream_sync(cfk_ctx *ctx, void *stream);
/* pinned host buffers */
int cfk_host_alloc(size_t bytes, void **out);
int cfk_host_free(void *ptr);

/* Number of kernels this context launched since creation (for accounting). */
long long cfk_kernel_launches(const cfk_ctx *ctx);

/* ---- allocation-free variant ------------------------------------------- */
/* No counterpart in the reference.  The local CFL step (dt_local and its grid
 * minimum, written to *dt_min_device) for callers that cannot call
 * cudaMalloc: a memory policy that forbids allocation after start-up (a pool
 * sized once), a framework that owns all device memory, or a time-critical
 * loop in which a cudaMalloc would synchronise the device.  It needs no context and allocates nothing: its scratch (one
 * partial minimum per 256-node row segment, ceil(mx/256)*my*mz <= 262144, i.e.
 * 2 MiB) is a file-scope device array that every GPU loading the library holds
 * until exit.  The first call on a device looks up that array's device address
 * (do it before any stream capture); after a cudaDeviceReset the next call
 * looks it up again.  The call makes param->device current while it launches
 * and restores the caller's current device before it returns.  Calls share
 * the scratch: calls that overlap on the GPU race.  Air model only; larger
 * zones are rejected with CFK_ERR_ARG and a message in err. */
int cfk_local_time_step_static(const cfk_param *param, const cfk_zone *zone, double *dt_min_device, void *stream,
                               char *err, size_t err_len);

/* ---- MLP chemistry surrogate ------------------------------------------- */
/* No counterpart in the reference: a learned replacement for the reaction
 * step of cfk_wu_reaction_step, trained on the device from trajectories of
 * the plain point-implicit integrator.
 *
 * Network: 12 standardised inputs (T, ln p, Box-Cox(Y_k) k=0..8, ln dt) ->
 * three tanh layers of 128 -> 11 outputs (Box-Cox increments of Y_k, dT,
 * ln of the reaction time scale after the step).  BF16 operands, FP32
 * accumulation on the tensor cores; everything after the network output
 * (inverse transform, element-conservation projection, energy-consistent
 * temperature, gate) is FP64.  Parameters: CFK_SG_NPARAM FP32 weights (four
 * row-major blocks W0 128x16, W1 128x144, W2 128x144, W3 16x144, biases in
 * column 15 of W0 and column 128 of the others) and CFK_SG_NNORM floats of
 * standardisation (in_mean[12], in_rstd[12], out_mean[11], out_std[11],
 * in_lo[12], in_hi[12], out_scale[11]); output j is learnt as
 * asinh(g_j / out_scale[j]) standardised (g_j itself where out_scale[j] = 0). */
#define CFK_SG_NPARAM 41216
#define CFK_SG_NNORM 81
#define CFK_SG_NIN 12
#define CFK_SG_NOUT 11

typedef struct cfk_surrogate_gate {
  double ood_margin;     /* allowed excursion beyond the training range (standardised units), on top of
                            1e-3 max(1, |training mean|) in the feature's own units */
  double dT_max;         /* |dT| per step (K) above which a node takes the plain integrator */
  double dT_consistency; /* |network dT - energy-consistent dT| (K) above which it does */
  double judge_tol_T;    /* judged node: |T_surrogate - T_plain| tolerance (K) */
  double judge_tol_bc;   /* judged node: max_k |bc(Y_surrogate) - bc(Y_plain)| tolerance (Box-Cox units) */
  double min_substeps;   /* nodes whose plain step would take fewer substeps (dt / reaction time scale)
                            stay on the plain integrator: cheap there, and accuracy-critical (induction) */
  int judge_stride;      /* every judge_stride-th node (rotating by step) also runs the plain integrator; 0 = off */
  int revert_steps;      /* steps a node that failed the judge stays on the plain integrator */
} cfk_surrogate_gate;

typedef struct cfk_surrogate_stats {
  long long cells, surrogate;
  long long fallback_ood, fallback_ignition, fallback_consistency, fallback_revert, fallback_newton, fallback_cheap;
  long long judged, judge_failed;
  double judge_max_dT, judge_mean_dT, judge_max_dbc;
} cfk_surrogate_stats;

/* Allocate (first call) and initialise the network: Xavier-uniform weights
 * from seed, zero biases, zero Adam moments.  elem_mu[n_elem][n_spec] holds
 * the element mass fractions per species (a_ek W_e / W_k) used by the
 * conservation projection; n_elem <= 4. */
int cfk_surrogate_init(cfk_ctx *ctx, unsigned long long seed, int n_elem, const double *elem_mu);
/* Training data from the plain integrator: phase 0 before a reaction step of
 * length dt snapshots every node's state (where the zone has a transport term
 * Cn, the states it alone reaches at the middle and the end of the step);
 * phase 1 after it writes one row per node (node order i fastest) of raw
 * features X[.][12] and targets G[.][11] (device float arrays). */
int cfk_surrogate_record(cfk_ctx *ctx, int phase, double dt, float *X, float *G, void *stream);
/* Standardisation from n rows of (X, G) on the device; the output scales
 * are the median |g_j| of a strided sample of the rows. */
int cfk_surrogate_fit_normalization(cfk_ctx *ctx, const float *X, const float *G, long long n);
/* Adam on the mean squared error of the standardised outputs: epochs passes
 * over n rows in minibatches of `batch` (a fresh pseudo-random row order per
 * epoch), learning rate cosine-annealed from lr0 to lr1.  loss_per_epoch
 * (host double[epochs], may be NULL) receives each epoch's mean loss. */
int cfk_surrogate_train(cfk_ctx *ctx, const float *X, const float *G, long long n, int epochs, int batch, double lr0,
                        double lr1, unsigned long long seed, double *loss_per_epoch);
/* Gradient of the mean loss over the n rows (device float[CFK_SG_NPARAM]),
 * and the loss itself (host, may be NULL); the weights are not changed. */
int cfk_surrogate_gradients(cfk_ctx *ctx, const float *X, const float *G, long long n, float *grad_out,
                            double *loss_out);
/* Standardised network outputs for n rows of raw features: Y (device
 * float[n][16], columns 11..15 are padding). */
int cfk_surrogate_forward(cfk_ctx *ctx, const float *X, long long n, float *Y);
/* Host copies of the FP32 weights (float[CFK_SG_NPARAM]) and standardisation
 * (float[CFK_SG_NNORM]); either pointer may be NULL. */
int cfk_surrogate_get_params(cfk_ctx *ctx, float *weights, float *norm);
int cfk_surrogate_set_params(cfk_ctx *ctx, const float *weights, const float *norm);
int cfk_surrogate_default_gate(cfk_surrogate_gate *gate);
/* Surrogate reaction step over dt at every node (constant volume; a bound Cn
 * is added after the reaction change).  Nodes outside the training range,
 * that the plain integrator would finish in fewer than min_substeps
 * substeps, with |dT| > dT_max, with an inconsistent network dT, whose
 * element-conservation projection or energy Newton iteration fails
 * (counted as fallback_newton), or that failed the judge within
 * revert_steps, are integrated by the plain FP64 work-queue kernel instead;
 * a rotating
 * 1/judge_stride of the remaining nodes is integrated by it as well and
 * compared with the surrogate's prediction.  stats (may be NULL) makes the
 * call synchronise the stream and report the counts. */
int cfk_surrogate_reaction_step(cfk_ctx *ctx, double dt, const cfk_surrogate_gate *gate, int step_index,
                                cfk_surrogate_stats *stats, void *stream);
/* cfk_wu_splitting_step whose reaction sub-step (the plain integrator with
 * the frozen transport term Cn, reference src/StrangSplitting.cu:475-502)
 * also writes one training row per node, as cfk_surrogate_record does around
 * a reactor step: the features are read at the state the frozen transport
 * term alone reaches half-way through the sub-step, the targets are the
 * changes from the state it reaches at the end.  X, G: device float arrays
 * of mx*my*mz rows.  Needs cfk_surrogate_init. */
int cfk_wu_splitting_step_record(cfk_ctx *ctx, int schedule, float *X, float *G, double *dt_used, void *stream);
/* cfk_wu_splitting_step with the gated surrogate as its reaction sub-step:
 * each node's change is predicted from its mid-sub-step transported state
 * and applied to its end-of-sub-step transported state (with Cn = 0 both are
 * the node's own state, as in cfk_surrogate_reaction_step); nodes the gate
 * or the judge send to the plain integrator integrate with the frozen Cn.
 * The transport half-steps are those of the plain step.  stats as in
 * cfk_surrogate_reaction_step. */
int cfk_wu_splitting_step_surrogate(cfk_ctx *ctx, const cfk_surrogate_gate *gate, int step_index,
                                    cfk_surrogate_stats *stats, double *dt_used, void *stream);

/* ---- measurement ------------------------------------------------------ */
/* Phases of a step timed with CUDA events when profiling is on (RK3 and Wu
 * steps; graph replays are not instrumented).  CFK_PH_REACTION is the
 * reaction sub-step of Wu's splitting (plain, recorded or surrogate). */
enum cfk_phase {
  CFK_PH_INVISCID = 0, CFK_PH_VISCOUS, CFK_PH_UPDATE, CFK_PH_BC, CFK_PH_PROPS, CFK_PH_DT, CFK_PH_REACTION,
  CFK_NPHASE
};
int cfk_set_profiling(cfk_ctx *ctx, int on);
/* Synchronises the recorded events, writes the summed milliseconds and kernel
 * counts per phase (arrays of CFK_NPHASE) and clears the record. */
int cfk_profile_read(cfk_ctx *ctx, double *ms, long long *kernels);
/* Achievable FP64 FMA throughput of the current device in TFLOP/s, measured
 * with a register-resident FMA chain kernel (the roofline denominator of the
 * FP64-bound kernels). */
int cfk_measure_fp64_peak(double *tflops);

#ifdef __cplusplus
}
#endif
#endif
