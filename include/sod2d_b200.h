/*
 * sod2d_b200 — B200-native (sm_100a) explicit spectral-element RHS of SOD2D, C ABI.
 *
 * Scope: the compressible Navier–Stokes right-hand side on HEX64 (p=3) elements with GLL
 * collocation (convection in skew-symmetric split form, viscous/heat/artificial diffusion,
 * entropy residual and entropy viscosity), the lumped-mass RK4 step that drives it, and the
 * incompressible pressure-Poisson PCG.  Every entry point below replaces one reference routine
 * or one reference call site, cited as file:line of the SOD2D sources.
 *
 * Conventions shared by all entry points:
 *  - Arrays keep the reference's Fortran column-major layouts (connec(nelem,nnode),
 *    He(ndime,ndime,ngaus,nelem), u(npoin,ndime), mu_e(nelem,ngaus) ...).  Node ids in
 *    connec and lpoin-style arrays are 1-based when index_base == 1 (Fortran callers) and
 *    0-based when index_base == 0.
 *  - "dev" pointers are device pointers (cudaMalloc / OpenACC deviceptr / torch tensors);
 *    "host" pointers are host memory (pageable or pinned).
 *  - Every function returns SOD_OK or a negative SOD_ERR_* code; sod_last_error() returns a
 *    thread-local message for the last failure.  Nothing aborts the process.
 *  - Work is stream-ordered on the cudaStream_t passed in (0 = legacy default stream).  A
 *    SodMesh handle must be used by one host thread at a time.
 *  - The precision argument selects SOD_FP64 (all arithmetic in FP64) or SOD_MIXED
 *    (element-local derivative and flux arithmetic in FP32 on deviation fields; nodal
 *    assembly, RK state, lumped mass and reductions in FP64).
 */
#ifndef SOD2D_B200_H
#define SOD2D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* sod_stream_t; /* a cudaStream_t */

enum {
  SOD_OK = 0,
  SOD_ERR_ARG = -1,           /* invalid argument (null pointer, bad size, bad layout)       */
  SOD_ERR_CUDA = -2,          /* a CUDA runtime call failed                                  */
  SOD_ERR_NONFINITE = -3,     /* a NaN/Inf was detected in the state or residual             */
  SOD_ERR_NOT_CONVERGED = -4, /* CG reached max_iter before the tolerance                    */
  SOD_ERR_TIMEOUT = -5,       /* a bounded host wait on device work expired                  */
  SOD_ERR_NOMEM = -6,         /* device allocation failed                                    */
  SOD_ERR_UNSUPPORTED = -7    /* option outside the implemented path (p != 3, LES ...)        */
};

typedef enum { SOD_FP64 = 0, SOD_MIXED = 1 } SodPrecision;

/* Physical and numerical parameters.  Defaults (sod_params_default) reproduce
 * mod_numerical_params.f90:8-99 and the TGV case of TGVSolver.f90:77-103. */
typedef struct {
  double gamma_gas;             /* TGVSolver.f90:92                                       */
  double Rgas;                  /* TGVSolver.f90:95, also nscbc_Rgas_inf (:102)           */
  double Cp;                    /* TGVSolver.f90:87                                       */
  double Prt;                   /* TGVSolver.f90:88                                       */
  double ce, cmax, cglob;       /* mod_numerical_params.f90:24-26                         */
  double c_rho, c_ener;         /* mod_numerical_params.f90:27-28                         */
  int32_t flag_normalise_entropy; /* mod_numerical_params.f90:23                          */
  double cfl_conv, cfl_diff;    /* CFDSolverBase cfl_conv / cfl_diff                      */
  int32_t flag_les;             /* 1: Vreman sgs_visc after each step (time_integ.f90:498-506) */
  double c_sgs;                 /* mod_numerical_params.f90:15 (0.025)                    */
  int32_t flag_total_enthalpy;  /* 1: convection by full_convec_ijk_H (time_integ.f90:361-365;
                                   mod_numerical_params.f90:20, default 0)                 */
} SodParams;

void sod_params_default(SodParams* p);

/* Mesh description handed to sod_mesh_create.  All arrays host, Fortran layouts.  The
 * geometry arrays (He, gpvol, Ml, helem, helem_l) are optional: when null they are computed
 * on the device from coord_orig/connec_orig exactly as the reference's setup does
 * (elem_jacobian jacobian_oper.f90:9-138, lumped_mass_spectral mass_matrix.f90:11-43,
 * char_length mod_geom.f90:13-37, char_length_spectral mod_geom.f90:39-66). */
typedef struct {
  int32_t nelem;             /* elements                                                 */
  int32_t npoin;             /* rows of the state arrays (unique nodes, or every lattice
                                point with periodic slave rows when lpoin_w is given)    */
  int32_t npoin_orig;        /* rows of coord_orig (nodes incl. periodic images)         */
  int32_t porder;            /* must be 3                                                */
  int32_t index_base;        /* 0 or 1                                                   */
  const int32_t* connec;     /* (nelem,64) connecParWork: unique node ids                */
  const int32_t* connec_orig;/* (nelem,64) connecParOrig: ids into coord_orig (optional) */
  const double* coord_orig;  /* (npoin_orig,3) (optional if geometry is given)           */
  const double* dlxigp_ip;   /* (64,3,4) 1-D Lagrange derivative table                   */
  const double* wgp;         /* (64) GLL weights                                          */
  const int32_t* invAtoIJK;  /* (4,4,4) local node of sod2d (i,j,k), index_base applies  */
  const int32_t* gmshAtoI;   /* (64) sod2d i of local node (1..4 or 0..3 by index_base)  */
  const int32_t* gmshAtoJ;
  const int32_t* gmshAtoK;
  const double* He;          /* (3,3,64,nelem) optional                                  */
  const double* gpvol;       /* (1,64,nelem)   optional                                  */
  const double* Ml;          /* (npoin)        optional                                  */
  const double* helem;       /* (nelem)        optional                                  */
  const double* helem_l;     /* (nelem,64)     optional                                  */
  /* Working nodes of rk_4_main's node loops (npoin_w, lpoin_w(npoin_w): workingNodesPar,
   * mod_mpi_mesh.f90:25-28; time_integ.f90:147,267-285,445-471).  lpoin_w = null: every row
   * works.  Otherwise the rows not listed are periodic slaves, as in SOD2D's mesh arrays
   * (coordPar with every lattice point, connecParWork with each image replaced by its master):
   * connec must reference exactly the listed rows, every step leaves the slave rows of the
   * state untouched (their mu_fluid is re-evaluated from their Tem, as sutherland_viscosity
   * runs over all npoin), and the entropy normalisation averages over the listed rows. */
  int32_t npoin_w;
  const int32_t* lpoin_w;    /* (npoin_w) index_base applies                             */
} SodMeshDesc;

typedef struct SodMesh SodMesh;

/* Upload a mesh, build the deterministic node->(element, local node) CSR gather map and the
 * device geometry.  Replaces the setup calls of CFDSolverBase_run (CFDSolverBase.f90:2115-2233:
 * evalJacobians :1280-1317, evalMass :1364-1389, evalCharLength :783-800) and the
 * `!$acc enter data` residency of init_rk4_solver (time_integ.f90:31-95). */
int sod_mesh_create(const SodMeshDesc* desc, const SodParams* params, SodMesh** out);
void sod_mesh_destroy(SodMesh* mesh);
/* Copy the device geometry back in the reference layouts (any pointer may be null). */
int sod_mesh_get_geometry(SodMesh* mesh, double* He, double* gpvol, double* Ml, double* helem,
                          double* helem_l);
/* Replace the parameters; step graphs captured with the old ones are dropped. */
int sod_mesh_set_params(SodMesh* mesh, const SodParams* params);

/* ---- Boundary conditions (non-periodic meshes: rk_4_main with noBoundaries = .false.) ---- */

/* The nscbc_* values read by temporary_bc_routine_dirichlet_prim (mod_bc_routines.f90:17-180). */
typedef struct {
  double rho_inf, u_inf, p_inf, c_inf; /* far-field state (bc_type_far_field = 1)          */
  double gamma_inf, Rgas_inf;          /* nscbc_gamma_inf, nscbc_Rgas_inf                   */
  double T_H, T_C;                     /* wall temperatures of codes 4 (hot) and 5 (cold)   */
} SodBcParams;

/* Register the boundary data rk_4_main takes (time_integ.f90:137-141) and switch the mesh's
 * step to the non-periodic path: host arrays of npoin rows, node ids in the mesh's
 * index_base.  bou_codes_nodes: a node is on a boundary when its code is below
 * max_num_bou_codes = 10 (mod_constants.f90:29; codes :41-48); lnbn_nodes: nearBoundaryNode
 * (mod_geom.f90:101-121), read for boundary nodes only; normalsAtNodes (npoin,3); u_buffer
 * (npoin,3), may be null (zeros).  Each step then applies temporary_bc_routine_dirichlet_prim
 * to every stage state and to the updated state, and bc_fix_dirichlet_residual_entropy to the
 * entropy residual (time_integ.f90:256-259,299-301,434-437,474-477).  bou_codes_nodes = null
 * removes the boundaries.  Captured step graphs of the mesh are dropped.  The ensemble
 * (sod_batch_*) rejects meshes with boundaries; sod_rk4_step_vjp differentiates through the
 * routines of every code. */
int sod_mesh_set_boundaries(SodMesh* mesh, const int32_t* bou_codes_nodes, const int32_t* lnbn_nodes,
                            const double* normalsAtNodes, const double* u_buffer, const SodBcParams* bc);

/* Penalisation buffer zone of rk_4_main (flag_buffer_on and flag_buffer_*,
 * mod_numerical_params.f90:50-74): a zone is enabled by its on_* flag; east/west act on x,
 * north/south on y, top/bottom on z; east, north and top cover coordinates above their minimum,
 * west, south and bottom those below it.  The state is relaxed towards (nscbc_rho_inf,
 * u_buffer rho, E_inf), E_inf = rho_inf u_inf^2 / 2 + p_inf / (gamma_inf - 1). */
typedef struct {
  int32_t on_east, on_west, on_north, on_south, on_top, on_bottom;
  double e_min, e_size, w_min, w_size, n_min, n_size, s_min, s_size, t_min, t_size, b_min, b_size;
  double rho_inf, u_inf, p_inf, gamma_inf;
} SodBufferParams;

/* flag_buffer_on = .true.: registers the zone (coord (npoin,3) and u_buffer (npoin,3) host
 * arrays in Fortran order; u_buffer may be null: zeros).  Each step then applies updateBuffer
 * (time_integ.f90:510-589) to every stage state (:251) and to the updated state (:429), before
 * the boundary routine; sod_rk4_step_vjp differentiates through it.  The zone factor of each
 * node is formed here once.  p = null removes the zone.  Captured step graphs of the mesh are
 * dropped; ensemble meshes (sod_batch_*) reject it. */
int sod_mesh_set_buffer(SodMesh* mesh, const SodBufferParams* p, const double* coord, const double* u_buffer);
/* updateBuffer on device arrays rho (npoin), q (npoin,3), E (npoin) with the registered zone
 * (no-op without one). */
int sod_update_buffer(SodMesh* mesh, double* rho, double* q, double* E, sod_stream_t stream);

/* The optional source_term argument of rk_4_main (time_integ.f90:187,326-330): a device array
 * (npoin,3) the mesh keeps a pointer to (caller-owned; its values may change between steps,
 * the pointer may not be freed while registered).  Every stage then adds
 * mom_source_const_vect (elem_source.f90:20-55), - sum over the node's elements of gpvol s =
 * - Ml s, to the momentum residual, inside the ordered node gather in FP64 (both precisions),
 * and so does sod_rhs.  null removes it.  A source term is constant in the state: the step
 * adjoint only sees it through the stage states.  Ensemble meshes reject it. */
int sod_mesh_set_source_term(SodMesh* mesh, const double* source_term);

/* Adjoint of temporary_bc_routine_dirichlet_prim in (rho, q, E): bar (the adjoint of the new
 * state, device rho (npoin), q (npoin,3), E (npoin)) is replaced in place by the adjoint of the
 * old state.  (rho, q, E) is the state the routine read (used by far-field nodes, whose new
 * state is the HLL state of their lnbn node; may be null without them).  No-slip walls zero the
 * rows they overwrite, outlet / ABL-top nodes pass through.  SOD_ERR_UNSUPPORTED for slip walls
 * (their new state reads a velocity this entry point is not given; sod_rk4_step_vjp handles
 * them) and for a far-field node whose lnbn node lies on a boundary. */
int sod_bc_dirichlet_prim_vjp(SodMesh* mesh, const double* rho, const double* q, const double* E,
                              double* bar_rho, double* bar_q, double* bar_E, sod_stream_t stream);

/* Wall model of rk_4_main (isWallModelOn, time_integ.f90:334-357): type 1 Reichardt
 * (evalWallModelReichardt, mod_wall_model.f90:12-175), 2 ABL (evalWallModelABL, :177-300; needs
 * walave_u, as the reference, and zo).  Host arrays in the reference layouts and the mesh's
 * index_base: bound (nboun,npbou=16), bounorm (nboun,3*npbou), wgp_b (npbou), listBoundsWM
 * (numBoundsWM faces), point2elem (npoin), coord (npoin,3), normalsAtNodes (npoin,3), zo (npoin)
 * or null; walave_u: a device (npoin,3) array the mesh keeps a pointer to (flag_walave), or null
 * for the stage velocity.  Each stage then adds the modelled wall shear to the momentum
 * residual of the wall nodes.  numBoundsWM = 0 removes the model.  The RHS and step adjoints
 * include it; the ensemble rejects meshes with a wall model. */
int sod_mesh_set_wall_model(SodMesh* mesh, int32_t type, int32_t nboun, int32_t npbou, const int32_t* bound,
                            const double* bounorm, const double* wgp_b, int32_t numBoundsWM,
                            const int32_t* listBoundsWM, const int32_t* point2elem, const double* coord,
                            const double* normalsAtNodes, const double* zo, const double* walave_u);
/* The registered wall model as the reference routine: Rdiff (npoin,3) += the wall shear terms from
 * device rho (npoin), u (npoin,3) (the exchange velocity: aux_u or walave_u) and mu_fluid
 * (npoin); tauw (npoin,3) receives tmag * tvelo, or may be null. */
int sod_wall_model(SodMesh* mesh, const double* rho, const double* u, const double* mu_fluid, double* Rdiff,
                   double* tauw, sod_stream_t stream);
/* tauw of the last evaluation of the wall model inside the library: a step's last stage, or the
 * forward recompute of a step adjoint (device (npoin,3)). */
int sod_wall_model_tauw(SodMesh* mesh, double* tauw, sod_stream_t stream);

/* Device-resident solver state in the reference's array layouts (level pos=2 only).
 * Every pointer is a device pointer owned by the caller. */
typedef struct {
  double* rho;      /* (npoin)    */
  double* q;        /* (npoin,3)  */
  double* E;        /* (npoin)    total energy rho*E */
  double* u;        /* (npoin,3)  output of the EOS update */
  double* pr;       /* (npoin)    */
  double* Tem;      /* (npoin)    */
  double* e_int;    /* (npoin)    */
  double* eta;      /* (npoin)    */
  double* csound;   /* (npoin)    */
  double* machno;   /* (npoin)    */
  double* mu_fluid; /* (npoin)    */
  double* mu_factor;/* (npoin)    input */
  double* mu_e;     /* (nelem,64) in: frozen entropy viscosity; out: updated */
  double* Reta;     /* (npoin)    out: -sum b_i Reta_i (time_integ.f90:467-471), may be null */
  double* mu_sgs;   /* (nelem,64) LES: in the step's frozen SGS viscosity, out updated by
                       sgs_visc (mod_sgs_viscosity.f90:13-125); null = no SGS (flag_les off) */
} SodState;

/* One explicit RK4 step: rk_4_main (time_integ.f90:137-508) on the compressible path
 * (either convection routine by flag_total_enthalpy, Sutherland on; LES when flag_les = 1 and state->mu_sgs is
 * set; boundary conditions when sod_mesh_set_boundaries registered some, else the periodic
 * noBoundaries path).  dt is read
 * from dt_dev (device double) so that a captured step needs no host value; when
 * update_dt != 0 the next dt from adapt_dt_cfl (mod_time_ops.f90:11-61) is written back to
 * dt_dev after the step (CFDSolverBase.f90:1592). */
int sod_rk4_main(SodMesh* mesh, SodState* state, const double* dt_dev, double* dt_next_dev,
                 SodPrecision prec, sod_stream_t stream);

/* nsteps steps of sod_rk4_main captured once into a CUDA graph per (mesh, state, precision)
 * and replayed; dt evolves on the device.  Returns after enqueueing. */
int sod_rk4_steps(SodMesh* mesh, SodState* state, double* dt_dev, int nsteps, SodPrecision prec,
                  sod_stream_t stream);

/* nsteps eager steps with CUDA events around every kernel; ms_out[0..2] receive the mean
 * duration of one fused-RHS launch, one gather/RK-stage launch and one entropy-viscosity+dt
 * launch.  Used for the live roofline figures. */
int sod_step_profile(SodMesh* mesh, SodState* state, double* dt_dev, int nsteps, SodPrecision prec,
                     sod_stream_t stream, float* ms_out);

/* Autotuner of the RK stage (no reference counterpart): times, on the given state, one RK stage
 * (fused RHS + gather / stage update into the library's stage buffers; the caller's arrays are
 * only read) for every configuration of two dimensions - elements per CTA {1,2,4,8} and the
 * launch shape: two launches per stage, or (on the periodic path) one cooperative launch per
 * stage with 1/2, 3/4 or all of the CTAs per SM that fit - 3 warm-up + 10 timed stages each, and
 * keeps the fastest for this mesh and precision; captured step graphs use it.  best_ms receives
 * the fastest fused-RHS launch alone; sod_autotune_table returns the whole sweep. */
int sod_autotune(SodMesh* mesh, SodState* state, SodPrecision prec, int* best_epb, float* best_ms,
                 sod_stream_t stream);
/* The last sweep of sod_autotune for a precision: up to cap rows of (elements per CTA, CTAs per
 * SM of the one-launch stage or 0 for two launches, ms per stage); returns the number of rows. */
int sod_autotune_table(SodMesh* mesh, SodPrecision prec, int cap, int32_t* epb, int32_t* ctas_per_sm,
                       float* ms_per_stage);
/* Pins the fused-RHS elements per CTA of a precision (1, 2, 4 or 8; 0: the default).  Captured
 * step graphs are dropped when it changes. */
int sod_set_rhs_config(SodMesh* mesh, SodPrecision prec, int config);
/* Pins the launch shape of an RK stage: 0 = two launches (fused RHS, then the gather); n > 0 =
 * one cooperative launch of min(n, what fits) resident CTAs per SM that runs the fused RHS over
 * element tiles, a grid barrier and the gather (and, at stage 4, the entropy viscosity and dt):
 * four launches per step.  Used on the periodic path only (without boundaries, buffer zone,
 * wall model, source term or LES the step falls back to two launches per stage). */
int sod_set_stage_launch(SodMesh* mesh, SodPrecision prec, int ctas_per_sm);

/* compute_fieldDerivs (mod_postpro.f90:12-139) on device arrays rho (npoin) and u (npoin,3):
 * gradRho (npoin,3), curlU (npoin,3) = sum_jk leviCivi(i,j,k) du_j/dx_k, divU (npoin) =
 * (div(rho u) + rho div u) / 2 and Qcrit (npoin) = -1/2 du_i/dx_j du_j/dx_i, each averaged over
 * the elements holding the node (lelpn).  leviCivi: host (3,3,3) Fortran array, or null for the
 * symbol CFDSolverBase sets (CFDSolverBase.f90:1248-1253). */
int sod_compute_field_derivs(SodMesh* mesh, const double* rho, const double* u, const double* leviCivi,
                             double* gradRho, double* curlU, double* divU, double* Qcrit, sod_stream_t stream);

/* Host-buffer variant of sod_rk4_main for the CPU-side drop-in (the reference's CPU build
 * calls rk_4_main on host arrays): copies rho,q,E,mu_e,mu_factor in, runs one step and copies
 * rho,q,E,u,pr,Tem,e_int,eta,csound,machno,mu_fluid,mu_e back.  dt_host in, dt_next_host out.
 * On a mesh with periodic slave rows (lpoin_w) the fields it copies back are also copied in, so
 * that their slave rows come back as they were.  The state fields are copied back on a stream
 * the mesh owns, which starts once the step has formed them; the call returns after every copy
 * has landed (pinned host arrays give the copies their full PCIe rate). */
int sod_rk4_main_host(SodMesh* mesh, SodState* host_state, double dt_host, double* dt_next_host,
                      SodPrecision prec, sod_stream_t stream);

/* Full RHS of one stage at a given conserved state, lumped-mass solved: what rk_4_main's
 * stage loop forms at time_integ.f90:266-393 (EOS, generic_scalar_convec_ijk, Sutherland,
 * full_diffusion_ijk, full_convec_ijk, sum, /Ml).  Outputs (npoin) / (npoin,3) device arrays. */
int sod_rhs(SodMesh* mesh, const double* rho, const double* q, const double* E,
            const double* mu_e, const double* mu_factor, double* Rmass, double* Rmom,
            double* Rener, double* Reta, SodPrecision prec, sod_stream_t stream);

/* smart_visc_spectral (mod_entropy_viscosity.f90:14-123) incl. the global entropy
 * normalisation and the convertIJK 3x3x3 filter (mod_filters.f90:15-55). */
int sod_smart_visc_spectral(SodMesh* mesh, const double* Reta, const double* rho, const double* u,
                            const double* csound, const double* Tem, const double* eta,
                            double* mu_e, sod_stream_t stream);

/* adapt_dt_cfl (mod_time_ops.f90:11-61) with both limits; result written to dt_dev. */
int sod_adapt_dt_cfl(SodMesh* mesh, const double* u, const double* csound, const double* mu_fluid,
                     const double* mu_sgs, const double* rho, double* dt_dev, sod_stream_t stream);

/* ---- Per-routine entry points with the reference argument lists (device arrays) -------- */

/* full_convec_ijk (elem_convec.f90:211-460); E is the energy-like field the caller passes
 * (enthalpy h in rk_4_main, time_integ.f90:364).  Outputs are overwritten. */
int sod_full_convec_ijk(SodMesh* mesh, const double* u, const double* q, const double* rho,
                        const double* pr, const double* E, double* Rmass, double* Rmom,
                        double* Rener, sod_stream_t stream);
/* full_convec_ijk_H (elem_convec.f90:20-208): the total-enthalpy form, energy flux (E + p) u;
 * E is the total energy rho E (time_integ.f90:362).  Outputs are overwritten. */
int sod_full_convec_ijk_H(SodMesh* mesh, const double* u, const double* q, const double* rho,
                          const double* pr, const double* E, double* Rmass, double* Rmom,
                          double* Rener, sod_stream_t stream);
/* generic_scalar_convec_ijk (elem_convec.f90:462-570). */
int sod_generic_scalar_convec_ijk(SodMesh* mesh, const double* q, const double* eta,
                                  const double* u, double* Rconvec, sod_stream_t stream);
/* full_diffusion_ijk (elem_diffu.f90:12-198); mu_sgs may be null (zero). */
int sod_full_diffusion_ijk(SodMesh* mesh, double Cp, double Pr, const double* rho_n,
                           const double* rho, const double* u, const double* Tem,
                           const double* mu_fluid, const double* mu_e, const double* mu_sgs,
                           double* Rmass, double* Rmom, double* Rener, sod_stream_t stream);
/* lumped_solver_scal / lumped_solver_vect (mod_solver.f90:23-58): R(:,c) /= Ml, ncomp 1 or 3. */
int sod_lumped_solver(SodMesh* mesh, double* R, int ncomp, sod_stream_t stream);
/* sutherland_viscosity (mod_fluid_viscosity.f90:21-41). */
int sod_sutherland_viscosity(int32_t npoin, const double* Tem, const double* mu_factor,
                             double* mu_fluid, sod_stream_t stream);

/* ---- The same routines with the reference's complete argument lists ---------------------
 * full_convec_ijk (elem_convec.f90:211-224), full_convec_ijk_H (:20-33),
 * generic_scalar_convec_ijk (:462-476), full_diffusion_ijk (elem_diffu.f90:12-25) and
 * smart_visc_spectral (mod_entropy_viscosity.f90:14-28): every argument of the Fortran
 * subroutine, in its order and layout, as a device pointer (the arrays SOD2D keeps resident),
 * with one addition, index_base, after npoin (1 for Fortran callers).  The mesh travels with
 * each call, as in the reference: the call builds a transient device view of it (element-major
 * connectivity and geometry, the ordered node->element gather map sorted on the device), runs
 * the handle-based routine's kernels on it (the results equal those of the entry points above
 * bit for bit), waits for the stream and releases the view.  It allocates per call; a time loop
 * creates a SodMesh once instead.  Arguments the routine does not read (Ngp, dNgp, xgp; Ml in
 * full_diffusion_ijk; Ngp, coord, dNgp, Ml and the scratch mue_l in smart_visc_spectral) are
 * accepted and ignored.  invAtoIJK, when given, must invert gmshAtoI/J/K (SOD_ERR_ARG otherwise);
 * node ids outside [index_base, index_base + npoin) give SOD_ERR_ARG.  smart_visc_spectral reads
 * the module variables of mod_numerical_params (ce, cmax, cglob, c_rho, c_ener,
 * flag_normalise_entropy) and nscbc_Rgas_inf from params (null: defaults); its lpoin_w must
 * list exactly the nodes connec references. */
int sod_full_convec_ijk_ref(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                            const double* Ngp, const double* dNgp, const double* He, const double* gpvol,
                            const double* dlxigp_ip, const double* xgp, const int32_t* invAtoIJK,
                            const int32_t* gmshAtoI, const int32_t* gmshAtoJ, const int32_t* gmshAtoK,
                            const double* u, const double* q, const double* rho, const double* pr, const double* E,
                            double* Rmass, double* Rmom, double* Rener, sod_stream_t stream);
int sod_full_convec_ijk_H_ref(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                              const double* Ngp, const double* dNgp, const double* He, const double* gpvol,
                              const double* dlxigp_ip, const double* xgp, const int32_t* invAtoIJK,
                              const int32_t* gmshAtoI, const int32_t* gmshAtoJ, const int32_t* gmshAtoK,
                              const double* u, const double* q, const double* rho, const double* pr, const double* E,
                              double* Rmass, double* Rmom, double* Rener, sod_stream_t stream);
int sod_generic_scalar_convec_ijk_ref(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                                      const double* Ngp, const double* dNgp, const double* He, const double* gpvol,
                                      const double* dlxigp_ip, const double* xgp, const int32_t* invAtoIJK,
                                      const int32_t* gmshAtoI, const int32_t* gmshAtoJ, const int32_t* gmshAtoK,
                                      const double* q, const double* eta, const double* u, double* Rconvec,
                                      sod_stream_t stream);
int sod_full_diffusion_ijk_ref(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                               const double* Ngp, const double* He, const double* gpvol, const double* dlxigp_ip,
                               const int32_t* invAtoIJK, const int32_t* gmshAtoI, const int32_t* gmshAtoJ,
                               const int32_t* gmshAtoK, double Cp, double Pr, const double* rho_n, const double* rho,
                               const double* u, const double* Tem, const double* mu_fluid, const double* mu_e,
                               const double* mu_sgs, const double* Ml, double* Rmass, double* Rmom, double* Rener,
                               sod_stream_t stream);
int sod_smart_visc_spectral_ref(int32_t nelem, int32_t npoin, int32_t npoin_w, int32_t index_base,
                                const int32_t* connec, const int32_t* lpoin_w, const double* Reta, const double* Ngp,
                                const double* coord, const double* dNgp, const double* gpvol, const double* wgp,
                                double gamma_gas, const double* rho, const double* u, const double* csound,
                                const double* Tem, const double* eta, const double* helem_l, const double* helem,
                                const double* Ml, double* mu_e, const int32_t* invAtoIJK, const int32_t* gmshAtoI,
                                const int32_t* gmshAtoJ, const int32_t* gmshAtoK, double* mue_l,
                                const SodParams* params, sod_stream_t stream);

/* Allocation-free full_convec_ijk, for callers that cannot allocate device memory: host codes
 * whose device memory is owned by the OpenACC runtime or by their own fixed pool (as SOD2D's
 * GPU build keeps its arrays in OpenACC present tables / managed memory) cannot create a
 * SodMesh, which allocates.  This entry point has no counterpart in the reference; it computes
 * what sod_full_convec_ijk / full_convec_ijk compute from the reference-layout device arrays
 * alone (connec(nelem,64), He(3,3,64,nelem), gpvol(1,64,nelem), dlxigp_ip(64,3,4),
 * gmshAtoI/J/K(64); ids index_base-based) and allocates nothing.  Its scratch (element
 * residuals and the node->element gather map, about 14 MB) is one static device array that
 * each GPU loading the library holds until exit, which limits a call to
 * SOD_NOALLOC_MAX_ELEM elements and 64*SOD_NOALLOC_MAX_ELEM nodes (larger: SOD_ERR_ARG).
 * All calls share that array: calls that overlap on the GPU race.  The first call on a
 * device looks up the array's address; make it before any stream capture.  The call waits
 * for its stream to finish (bounded by sod_set_wait_timeout) so it can report bad node ids
 * (SOD_ERR_ARG); on a stream that is capturing it enqueues nothing and returns
 * SOD_ERR_UNSUPPORTED, since that wait is not allowed there. */
#define SOD_NOALLOC_MAX_ELEM 4096
int sod_full_convec_ijk_noalloc(int32_t nelem, int32_t npoin, int32_t index_base, const int32_t* connec,
                                const double* He, const double* gpvol, const double* dlxigp_ip,
                                const int32_t* gmshAtoI, const int32_t* gmshAtoJ, const int32_t* gmshAtoK,
                                const double* u, const double* q, const double* rho, const double* pr,
                                const double* E, double* Rmass, double* Rmom, double* Rener,
                                sod_stream_t stream);

/* ---- Ensemble batching: many independent periodic meshes in one launch per stage -------
 * The reference runs ensembles as separate MPI applications (mod_mpi.f90:39-51,
 * TGVMultiSolver.f90:30-60); here the members are concatenated into one block-diagonal mesh
 * so each RK stage is one fused-RHS and one gather launch over all members and a step is one
 * CUDA graph.  Per member: its own state, Reynolds number (mu_factor), dt, entropy
 * normalisation and CFL limit.  The batch copies what it needs from the member meshes. */
typedef struct SodBatch SodBatch;
int sod_batch_create(SodMesh* const* meshes, int nmesh, SodBatch** out);
void sod_batch_destroy(SodBatch* B);
/* Host arrays of one member in the reference layouts: rho, q(N_i,3), E, mu_factor and
 * mu_e(E_i,64) are required; u(N_i,3), csound, mu_fluid are used by sod_batch_adapt_dt. */
int sod_batch_set_member(SodBatch* B, int member, const SodState* host);
/* Copy any non-null field of one member back to host arrays (reference layouts). */
int sod_batch_get_member(SodBatch* B, int member, SodState* host);
int sod_batch_set_dt(SodBatch* B, const double* dt_host);   /* [nmember] */
int sod_batch_get_dt(SodBatch* B, double* dt_host);         /* [nmember] */
/* adapt_dt_cfl (mod_time_ops.f90:11-61) per member from the members' u, csound, mu_fluid, rho. */
int sod_batch_adapt_dt(SodBatch* B, sod_stream_t stream);
/* The concatenated mesh (for sod_autotune and diagnostics; owned by the batch). */
int sod_batch_mesh(SodBatch* B, SodMesh** mesh);
/* sod_autotune on the concatenated ensemble state. */
int sod_batch_autotune(SodBatch* B, SodPrecision prec, int* best_epb, float* best_ms, sod_stream_t stream);
/* nsteps RK4 steps of every member, each step one captured graph; dt evolves per member. */
int sod_batch_rk4_steps(SodBatch* B, int nsteps, SodPrecision prec, sod_stream_t stream);

/* ---- Incompressible pressure Poisson (lib_sod2d_incomp) --------------------------------- */

typedef struct SodPoisson SodPoisson;
/* Set up the pinned pressure Laplacian that eval_laplacian_mult (mod_operators.f90:20-128)
 * applies matrix-free: the per-gauss-point metric gpvol He^T He (FP64 and an FP32 copy, 6
 * values per point) and the Jacobi diagonal of eval_laplacian_diag (:417-461); pinned node =
 * node 0 (lpoin_w(1), mod_operators.f90:46-48,125-127).  The handle keeps a pointer to the
 * mesh, which must outlive it. */
int sod_poisson_create(SodMesh* mesh, SodPoisson** out);
void sod_poisson_destroy(SodPoisson* P);
/* y = K x, matrix-free (device arrays of npoin): eval_laplacian_mult, x(pin) read as 0 and
 * y(pin) = 0. */
int sod_poisson_apply(SodPoisson* P, const double* x, double* y, sod_stream_t stream);
/* Jacobi diagonal (device array of npoin): eval_laplacian_diag. */
int sod_poisson_diag(SodPoisson* P, double* d, sod_stream_t stream);
/* conjGrad_pressure_incomp (mod_solver_incomp.f90:247-434): R holds the right-hand side on
 * entry and x0+x on exit; Rp0 is the initial guess; stops at ||r|| < tol ||r0||, with
 * beta = <r, z - z_old>/<r_old, z_old> as the reference; the stop test runs on the device and
 * the host reads the scalars every 16 iterations.  mixed != 0 runs FP32 Jacobi-PCG sweeps
 * (FP32 metric and vectors) inside FP64 residual iterative refinement.  Calls on one handle
 * must not overlap (its work vectors are shared).  Returns
 * SOD_ERR_NOT_CONVERGED when max_iter is reached first.  iters/final_rel may be null. */
int sod_conjgrad_pressure(SodPoisson* P, const double* Rp0, double* R, int max_iter, double tol,
                          int mixed, int* iters, double* final_rel, sod_stream_t stream);

/* ---- Boundary routines on device arrays (the mesh's registered boundary data) ---------- */
/* temporary_bc_routine_dirichlet_prim (mod_bc_routines.f90:17-180) in place on rho, q, u, pr,
 * E (npoin / (npoin,3) device arrays): every boundary node takes the far-field HLL state, the
 * no-slip wall state or the slip projection of its code, from the state of its lnbn node; u
 * is read (slip walls) and written, pr written for far-field nodes, as the reference. */
int sod_bc_dirichlet_prim(SodMesh* mesh, double* rho, double* q, double* u, double* pr, double* E,
                          sod_stream_t stream);
/* bc_fix_dirichlet_residual (mod_bc_routines.f90:181-221): zero Rmass, Rmom (and Rener for the
 * isothermal walls) on no-slip nodes. */
int sod_bc_fix_dirichlet_residual(SodMesh* mesh, double* Rmass, double* Rmom, double* Rener, sod_stream_t stream);
/* bc_fix_dirichlet_residual_entropy (mod_bc_routines.f90:265-291): zero R on no-slip nodes. */
int sod_bc_fix_dirichlet_residual_entropy(SodMesh* mesh, double* R, sod_stream_t stream);

/* ---- Taylor-Green diagnostics ------------------------------------------------------------ */
/* volAvg_EK and visc_dissipationRate (mod_analysis.f90:10-144), as the time loop calls them
 * (CFDSolverBase.f90:1413-1414): u(npoin,3), rho, mu_fluid (npoin), mu_e(nelem,64) device
 * arrays; rho0 = nscbc_rho_inf, volT = the domain volume (<= 0: the sum of gpvol, as the
 * reference's VolTot, CFDSolverBase.f90:1300-1312); out_dev (device, 5 doubles) receives EK,
 * eps_S, eps_D, eps_T and the volume used.  Sums are in a fixed order (deterministic). */
int sod_tgv_diagnostics(SodMesh* mesh, const double* rho, const double* u, const double* mu_fluid,
                        const double* mu_e, double rho0, double volT, double* out_dev,
                        sod_stream_t stream);

/* ---- Adjoint (reverse mode) of the RHS and of one RK4 step ------------------------------ */
/* No counterpart in the reference (SOD2D has no adjoint); these differentiate the FP64 path of
 * sod_rhs / sod_rk4_main with the entropy viscosity mu_e (and dt, and the LES mu_sgs of the
 * step) frozen at the given values, Sutherland's law differentiated.  All arrays are device arrays in the
 * SodState layouts (q and its adjoints: 3 columns of npoin). */

/* VJP of the stage RHS of sod_rhs (Rmass, Rmom, Rener, already divided by Ml): given seeds
 * (bar_Rmass, bar_Rmom, bar_Rener) writes grad = (dR/d(rho,q,E))^T seed (overwritten). */
int sod_rhs_vjp(SodMesh* mesh, const double* rho, const double* q, const double* E,
                const double* mu_e, const double* mu_factor, const double* bar_Rmass,
                const double* bar_Rmom, const double* bar_Rener, double* grad_rho, double* grad_q,
                double* grad_E, sod_stream_t stream);
/* sod_rk4_main that also writes its stage states Y2, Y3, Y4 to stages (device, 15*npoin
 * doubles: 3 stages x (rho, q x3, E) columns, FP64 in both precisions) for sod_rk4_step_vjp. */
int sod_rk4_main_record(SodMesh* mesh, SodState* state, const double* dt_dev, double* dt_next_dev,
                        double* stages, SodPrecision prec, sod_stream_t stream);
/* VJP of one RK4 step y_{n+1} = y_n - dt sum_s b_s R(Y_s) (rk_4_main, time_integ.f90:288-426)
 * at the state (rho, q, E) with mu_e, mu_sgs and dt_dev frozen: out = (dy_{n+1}/dy_n)^T bar.
 * mu_sgs (nelem,64): the step's SGS viscosity when flag_les = 1 (rho mu_sgs in the stress and
 * Cp/0.9 rho mu_sgs in the heat flux, differentiated through rho), null otherwise.  stages
 * from sod_rk4_main_record, or null to recompute them; out may alias bar.  On a mesh with
 * boundaries the map includes temporary_bc_routine_dirichlet_prim on every stage state and on
 * the update; for the no-slip codes 3-5 the routine is affine (constants on rho, q and, for
 * 4 and 5, E) and the outlet / ABL-top codes 2 and 8 leave the node alone, so its adjoint is a
 * constant mask of the wall rows; far-field nodes (code 1) take the HLL state of their lnbn
 * node, whose Jacobian is evaluated at the stage states and at the updated state (one more RHS
 * evaluation at the last stage state); slip walls (codes 6, 7) also read a velocity: zero at
 * stage 1, q/rho of the previous post-routine stage state at stages 2-4, and u(pos) of the input
 * state at the update, which the map takes as q/rho of (rho, q, E) (its value in every state a
 * step produces).  A registered wall model is differentiated too (its law by dual numbers). */
int sod_rk4_step_vjp(SodMesh* mesh, const double* rho, const double* q, const double* E,
                     const double* mu_e, const double* mu_sgs, const double* mu_factor,
                     const double* dt_dev, const double* stages, const double* bar_rho,
                     const double* bar_q, const double* bar_E, double* out_rho, double* out_q,
                     double* out_E, sod_stream_t stream);

/* ---- Legacy unit-test API ----------------------------------------------------------- */

/* CSR_SpMV_scal (legacy API pinned by unitt/unitt_CSR_SPMV_scal/unitt_CSR_SPMV_scal.f90:14-52):
 * u = Mc v, rdom 0-based row offsets (npoin+1), cdom 1-based columns.  Device arrays. */
int sod_csr_spmv_scal(int32_t npoin, int32_t nzdom, const int32_t* rdom, const int32_t* cdom,
                      const double* Mc, const double* v, double* u, sod_stream_t stream);

/* Legacy element-loop routines of the unit tests (names and argument lists from their call
 * sites: unitt/unitt_mass_convec/unitt_mass_convec.f90:151, unitt_mom_convec.f90:151,
 * unitt_ener_convec.f90:151, unitt_generic_scalar_convec.f90:151, unitt_mom_diffu.f90:148;
 * the routines themselves are no longer in src/).  Generic elements given by the caller's
 * tables: connec(nelem,nnode) 1-based, Ngp(ngaus,nnode), gpcar(ndime,nnode,ngaus,nelem),
 * gpvol(1,ngaus,nelem); ndime 2 or 3, nnode and ngaus <= 64; device arrays.  Residuals
 * R_a = sum_g gpvol N_a div(flux) with the flux formed at the nodes (the unit tests' .m
 * scripts): mass/generic q; momentum q_i u + p e_i (R(npoin,ndime)); energy u (E + p).
 * mom_diffusion: R_a,i = sum_g gpvol sum_j gpcar(j,a) tau_ij, tau = mu_e(elem)(grad u +
 * grad u^T - 2/3 div u I) (R(npoin,ndime), mu_e(nelem)).  Outputs are overwritten. */
int sod_legacy_mass_convec(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode, int32_t ndime,
                           const int32_t* connec, const double* Ngp, const double* gpcar,
                           const double* gpvol, const double* q, double* R, sod_stream_t stream);
int sod_legacy_generic_scalar_convec(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode,
                                     int32_t ndime, const int32_t* connec, const double* Ngp,
                                     const double* gpcar, const double* gpvol, const double* q,
                                     double* R, sod_stream_t stream);
int sod_legacy_mom_convec(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode, int32_t ndime,
                          const int32_t* connec, const double* Ngp, const double* gpcar,
                          const double* gpvol, const double* u, const double* q, const double* pr,
                          double* R, sod_stream_t stream);
int sod_legacy_ener_convec(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode, int32_t ndime,
                           const int32_t* connec, const double* Ngp, const double* gpcar,
                           const double* gpvol, const double* u, const double* pr, const double* E,
                           double* R, sod_stream_t stream);
int sod_legacy_mom_diffusion(int32_t nelem, int32_t ngaus, int32_t npoin, int32_t nnode, int32_t ndime,
                             const int32_t* connec, const double* Ngp, const double* gpcar,
                             const double* gpvol, const double* u, const double* mu_e, double* R,
                             sod_stream_t stream);

/* ---- Diagnostics ------------------------------------------------------------------------ */
const char* sod_last_error(void);
const char* sod_version(void);
/* Number of kernels this library enqueued since load (for launch accounting). */
int64_t sod_launch_count(void);
/* Failure detection.  Every step checks its new rho, q and E on the device (one predicate per
 * node in the update kernel) and raises a flag on a NaN/Inf; sod_check_finite waits for the
 * stream's work, returns SOD_ERR_NONFINITE when the flag is up (steps since the last check) and
 * clears it.  sod_rk4_main_host checks after its own step. */
int sod_check_finite(SodMesh* mesh, sod_stream_t stream);
/* Limit (seconds, 0 = none, the default) on the library's host waits for device work (the
 * synchronous entry points: sod_rk4_main_host, sod_conjgrad_pressure, sod_check_finite);
 * past it they return SOD_ERR_TIMEOUT and leave the queued work to complete on its own. */
void sod_set_wait_timeout(double seconds);

#ifdef __cplusplus
}
#endif
#endif /* SOD2D_B200_H */
