/*
 * atjup_gpu.h -- C ABI of the B200 (sm_100a) implementation of ATJUP's time-step hot path.
 *
 * The reference (RogerGrundmann/ATJUP) runs its time step as member functions of the singleton
 * cJupiterModel, on jagged `double***` arrays (lib/Array.h:25-31), with ~200 ATJUP_* environment
 * knobs read into function-local statics. This header replaces those call sites with plain
 * extern "C" entry points: the device owns the authoritative state (structure of arrays, phi
 * contiguous and padded), the host resolves every knob once into AtjupParams, and each entry
 * point returns an int status. Every function below names the reference routine it replaces.
 *
 * Layout of a 3-D field on the host side of this ABI: either a contiguous block of
 * im*jm*km doubles in (i, j, k) order with k fastest (i = radius, j = colatitude, k = longitude),
 * or the reference's own `double***` (x[i][j] is a row of km doubles).
 *
 * Thread safety: one context per model; calls on one context must not overlap. All work is
 * stream-ordered on the context's stream; entry points return after the work is enqueued unless
 * they return a host value (download, stats), which synchronises the stream.
 */
#ifndef ATJUP_GPU_H
#define ATJUP_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATJUP_ABI_VERSION 2

/* ---- status codes ---- */
enum {
    ATJUP_OK = 0,
    ATJUP_ERR_ARG = 1,            /* bad argument (null pointer, unknown id, size mismatch)  */
    ATJUP_ERR_UNSUPPORTED = 2,    /* a knob value this implementation does not provide       */
    ATJUP_ERR_CUDA = 3,           /* a CUDA runtime error; see atjup_gpu_last_error()          */
    ATJUP_ERR_NOT_CONVERGED = 4,  /* iterative solve hit its iteration cap                    */
    ATJUP_ERR_NONFINITE = 5,      /* a NaN/Inf census found non-finite values                 */
    ATJUP_ERR_NO_DEVICE = 6       /* no CUDA device, or the device is not sm_100              */
};

/* ---- field ids (upload / download / filter targets) ---- */
enum {
    ATJUP_F_T = 0, ATJUP_F_U, ATJUP_F_V, ATJUP_F_W,          /* prognostic dynamics           */
    ATJUP_F_P_DYN, ATJUP_F_P_HYDRO, ATJUP_F_P_STAT,           /* pressures                     */
    ATJUP_F_RHO_MIX, ATJUP_F_WALL_NUE, ATJUP_F_NUE,           /* frozen per-cell inputs        */
    ATJUP_F_AUX_U, ATJUP_F_AUX_V, ATJUP_F_AUX_W,              /* projection source (persist)   */
    ATJUP_F_P_BARO,                                           /* frozen geo-balance rest       */
    ATJUP_F_Q_RAD, ATJUP_F_Q_PRECIP,                          /* heating inputs                */
    ATJUP_F_H2O, ATJUP_F_H2O_CLOUD, ATJUP_F_H2O_ICE,          /* condensable species [kg/m3]   */
    ATJUP_F_NH3, ATJUP_F_NH3_CLOUD, ATJUP_F_NH3_ICE,          /* (vapour, cloud, ice per gas)  */
    ATJUP_F_CH4, ATJUP_F_CH4_CLOUD, ATJUP_F_CH4_ICE,
    ATJUP_F_H2S, ATJUP_F_NH4SH,                               /* chemistry species [kg/m3]     */
    ATJUP_F_TKE, ATJUP_F_DIS,                                 /* turbulence k*, omega* (or eps)*/
    ATJUP_F_S_PRECIP_H2O, ATJUP_F_S_PRECIP_H2O_CLOUD, ATJUP_F_S_PRECIP_H2O_ICE,
    ATJUP_F_S_PRECIP_NH3, ATJUP_F_S_PRECIP_NH3_CLOUD, ATJUP_F_S_PRECIP_NH3_ICE,
    ATJUP_F_S_PRECIP_CH4, ATJUP_F_S_PRECIP_CH4_CLOUD, ATJUP_F_S_PRECIP_CH4_ICE,
                                                              /* frozen microphysics sources   */
    ATJUP_F_MASSFLUX_H2S, ATJUP_F_MASSFLUX_NH3, ATJUP_F_MASSFLUX_NH4SH,
    ATJUP_F_FLUXLIM_NH4SH,                                    /* frozen chemistry sources      */
    ATJUP_F_PROD, ATJUP_F_TKE_SOURCE, ATJUP_F_DIS_SOURCE,     /* closure diagnostics (out)     */
    ATJUP_F_DIFFLUX_H2S, ATJUP_F_DIFFLUX_NH3, ATJUP_F_DIFFLUX_NH4SH,
                                                              /* diffusive chemistry fluxes    */
    ATJUP_F_CORIOLIS_FORCE, ATJUP_F_CENTRIFUGAL_FORCE, ATJUP_F_BUOYANCY_FORCE,
    ATJUP_F_PRESGRAD_FORCE, ATJUP_F_Q_LATENT, ATJUP_F_Q_SENSIBLE,
                                                              /* output diagnostics (out)      */
    ATJUP_F_COUNT
};

/* 2-D (jm x km) fields: the friction velocity of the k-epsilon wall term (Turbulence.h:336-377) */
enum { ATJUP_F2_VEL_STAR = 0, ATJUP_F2_COUNT };

/* ---- solver modes for atjup_gpu_pressure_solve ---- */
enum {
    ATJUP_SOLVE_SWEEPS = 0,    /* the reference: n red-black Gauss-Seidel sweeps, no residual   */
    ATJUP_SOLVE_RESIDUAL = 1,  /* same discrete operator, iterated to a relative residual       */
    ATJUP_SOLVE_SOR = 2        /* same operator by point red-black SOR with opts->omega, up to   */
                               /* max_iter sweeps, the residual checked every 50 sweeps; returns */
                               /* ATJUP_ERR_NOT_CONVERGED (stats filled) at the sweep cap        */
};
enum { ATJUP_PREC_FP64 = 0, ATJUP_PREC_MIXED = 1 };

/*
 * Every knob that changes a branch of the hot path, resolved on the host (the reference reads
 * them from the environment at first use; the values noted are the reference defaults).
 * atjup_params_default() fills this block with those defaults for the 41x181x361 grid.
 */
typedef struct AtjupParams {
    int32_t abi_version;               /* = ATJUP_ABI_VERSION                                   */
    int32_t im, jm, km;                /* 41, 181, 361 (cJupiterModel.h:166)                   */
    double dr, dthe, dphi;             /* 0.025, 1 deg, 1 deg (cJupiterModel.cpp:172-174)      */
    double dt;                         /* ATJUP_DT 0.005 (cJupiterModel.cpp:106)                */
    /* model constants (param.py / cJupiterDefaults.cpp.inc and ThermalPropertiesJup)          */
    double re, pr, g, omega, u_0, t_ref, L_atm;
    double r_mix, R_mix, cp_mix;
    double Coriolis, centrifugal, buoyancy;
    /* resolved knobs of RHS_Jup_Turb.cpp / RungeKutta_Jup_Turb.cpp                            */
    double sinthe_min;                 /* ATJUP_SINTHE_MIN 0.55 (cJupiterModel.h:1121)          */
    double p_dyn_to_bar;               /* r_mix u_0^2 1e-5 with ATJUP_PDYN_UNITS (h:1161)       */
    double t_diff_scale;               /* ATJUP_T_DIFF_SCALE 0.01 (cJupiterModel.h:268)         */
    double nd_cor, nd_cent, nd_buoy;   /* body-force scales (RHS_Jup_Turb.cpp:323-346)          */
    double buoy_scale, buoy_ramp;      /* ATJUP_BUOY_SCALE 1, ramp factor for this iteration   */
    double pgrad_scale;                /* ATJUP_PGRAD_SCALE 1                                   */
    double rad_coupling;               /* ATJUP_RAD_COUPLING 1                                  */
    double precip_coupling;            /* ATJUP_PRECIP_COUPLING 1                               */
    double turb_coupling;              /* ATJUP_TURB_COUPLING 1                                 */
    int32_t pgrad_wall, pgrad_wrap;    /* 1, 1 (RHS_Jup_Turb.cpp:103-117)                       */
    int32_t adiabatic, adiabatic_rho;  /* 1, 1 (RHS_Jup_Turb.cpp:459-474)                       */
    int32_t metric_split;              /* ATJUP_METRIC_SPLIT 1 (cJupiterModel.h:830)            */
    int32_t coriolis_split;            /* ATJUP_CORIOLIS_SPLIT 1 and metric_split (h:837)       */
    int32_t hydro_split;               /* ATJUP_HYDRO_SPLIT / ATJUP_NONDIM, 0                   */
    int32_t cell_hold;                 /* ATJUP_CELL_HOLD (follows geo balance), 1              */
    int32_t precip_rho_local;          /* ATJUP_PRECIP_RHO_LOCAL 1                              */
    int32_t local_rho;                 /* ATJUP_LOCAL_RHO 1                                     */
    int32_t rho_pdyn;                  /* ATJUP_RHO_PDYN (0 with geo balance)                   */
    int32_t has_nue;                   /* nue field non-zero (turbulence closure on)            */
    int32_t has_heating;               /* Q_rad / Q_precip fields present                       */
    /* pressure solver (PressureSolver.h:144-766)                                               */
    double p_dyn_cap;                  /* ATJUP_PDYN_CAP 0.2                                    */
    int32_t press_wall;                /* ATJUP_PRESS_WALL 1 (has_obstacle)                     */
    int32_t rigid_lid;                 /* ATJUP_BC_RIGID_LID 1                                  */
    int32_t press_sweeps;              /* ATJUP_PRESS_SWEEPS 1                                  */
    /* boundary conditions (BoundaryConditions.h, BC_Jup.h)                                     */
    int32_t top_taper;                 /* ATJUP_BC_TOP_TAPER 3                                  */
    int32_t lid_u;                     /* ATJUP_BC_LID_U = rigid lid, 1                         */
    int32_t pole_fill_rows;            /* 2 with ATJUP_BC_POLE_FILL 1                           */
    int32_t mount_t_ambient;           /* ATJUP_MOUNT_T_AMBIENT 1                               */
    /* per-iteration filters and glue (cJupiterModel.cpp:1328-1354)                             */
    int32_t shapiro_inloop;            /* ATJUP_VEL_SHAPIRO_INLOOP passes (0 = off)             */
    double shapiro_strength;           /* ATJUP_SHAPIRO_STRENGTH 1                              */
    int32_t v_massbal_stride;          /* ATJUP_V_MASSBAL_STRIDE 1                              */
    int32_t v_massbal_zonal;           /* ATJUP_V_MASSBAL_ZONAL (follows ATJUP_VORTEX), 1       */
    int32_t precision;                 /* the RK step: ATJUP_PREC_FP64, or ATJUP_PREC_MIXED: the    */
                                       /* stage inputs and accumulators of the 17 fields in FP32,  */
                                       /* the species and closure right-hand sides in FP32; the    */
                                       /* time-level-n state, the final update, the dynamics RHS,  */
                                       /* the pressure, the level means, the column balance and    */
                                       /* the loop's physics stay FP64                              */
    /* the in-loop projection around the obstacle (InitValues_Jup.cpp:1595-1822, called at      */
    /* cJupiterModel.cpp:1356-1363 after the column balance of v)                              */
    int32_t cone_proj_stride;          /* ATJUP_CONE_PROJ_STRIDE 10 (0 = off)                    */
    int32_t cone_proj_margin;          /* ATJUP_CONE_PROJ_MARGIN 40: box cells beyond the body   */
    int32_t cone_proj_div;             /* ATJUP_CONE_PROJ_DIV 3: H of the divergence solve       */
} AtjupParams;

typedef struct AtjupSolveOpts {
    int32_t mode;          /* ATJUP_SOLVE_SWEEPS or ATJUP_SOLVE_RESIDUAL                         */
    int32_t sweeps;        /* SWEEPS: number of red-black sweeps                                  */
    int32_t max_iter;      /* RESIDUAL: iteration cap (returns ATJUP_ERR_NOT_CONVERGED at it)     */
    int32_t precision;     /* RESIDUAL: ATJUP_PREC_FP64, or MIXED = the preconditioner in FP32     */
                           /* under FP64 Krylov vectors and FP64 iterative refinement             */
    double rel_tol;        /* RESIDUAL: target ||b - A p|| / ||b|| (y-weighted, fluid cells)      */
    double omega;          /* relaxation factor of the sweeps (reference: 1.0)                    */
    int32_t external_rhs;  /* RESIDUAL: 1 = solve A p = b for b in atjup_gpu_set_solve_rhs       */
} AtjupSolveOpts;

typedef struct AtjupSolveStats {
    int32_t iterations;    /* sweeps or Krylov iterations performed                              */
    int32_t inner_solves;  /* MIXED: FP32 inner solves under the FP64 refinement loop            */
    double rel_residual;   /* final ||b - A p|| / ||b||, or -1 when not computed (SWEEPS)       */
    double b_norm;         /* ||b|| of the projected right-hand side                              */
    double rel_floor;      /* eps * || |A| |p| || / ||b||: the rounding floor of the relative     */
                           /* residual of an FP64 p (RESIDUAL); the solve counts as converged at  */
                           /* rel_tol or, when rel_tol is below the floor, at <= 8 floor          */
} AtjupSolveStats;

typedef struct AtjupCtx AtjupCtx;

/* Defaults of the reference for the 41x181x361 grid (values noted in AtjupParams). */
void atjup_params_default(AtjupParams* p);

/* Create a device context: allocates the SoA state on the current CUDA device.
 * Replaces the field allocation of cJupiterModel::resetArrays (cJupiterModel.cpp:1570-1753). */
int atjup_gpu_create(const AtjupParams* params, AtjupCtx** out);
int atjup_gpu_destroy(AtjupCtx* ctx);

/* Use a caller-owned cudaStream_t (passed as void*); NULL = the context's own stream. */
int atjup_gpu_set_stream(AtjupCtx* ctx, void* stream);
/* The cudaStream_t (as void*) the context issues its work on, its own or the one set above, for
 * a caller that records events on it or orders its own work after the library's. Besides it the
 * library uses up to three streams of its own (the scalar stages of the RK step, and the two copy
 * streams of the asynchronous exchange). A process whose streams outnumber
 * CUDA_DEVICE_MAX_CONNECTIONS (8 by default) shares hardware queues between streams, which can
 * order an asynchronous copy behind unrelated compute. (No reference counterpart.) */
int atjup_gpu_stream(AtjupCtx* ctx, void** stream);

/* Geometry and frozen per-(i,j) inputs:
 *   rad[im]      metric radius rad.z (cJupiterModel.cpp:441-468 shifts it to R/L_atm + i dr)
 *   the[jm]      colatitude the.z
 *   solid[im*jm*km]  SeaMount mask (1 = solid), BC_Jup.h:353-458
 *   i_topo[jm*km]    first fluid level per column (i_topography)
 *   cell_vbar0 / cell_ubar0 [im*jm]  ATJUP_CELL_HOLD means (may be NULL when cell_hold = 0)   */
int atjup_gpu_set_grid(AtjupCtx* ctx, const double* rad, const double* the,
                       const uint8_t* solid, const int32_t* i_topo,
                       const double* cell_vbar0, const double* cell_ubar0);

/* Copy a contiguous (i,j,k) host field to / from the device (synchronous).
 * Replaces the host Array as the owner of that field. */
int atjup_gpu_upload(AtjupCtx* ctx, int32_t field_id, const double* host);
int atjup_gpu_download(AtjupCtx* ctx, int32_t field_id, double* host);
/* The same for the reference's jagged Array storage (x[i][j] -> km doubles). */
int atjup_gpu_upload_array(AtjupCtx* ctx, int32_t field_id, double*** x);
int atjup_gpu_download_array(AtjupCtx* ctx, int32_t field_id, double*** x);

/* Device pointer of a field (row pitch in elements via *pitch) for zero-copy interop (DLPack). */
int atjup_gpu_field_ptr(AtjupCtx* ctx, int32_t field_id, void** dev_ptr, int32_t* pitch);

/* Asynchronous exchange of whole fields, for a caller that keeps the state on the host and hands it
 * to the library every step (no counterpart in the reference, which has no device). The copies run
 * on two copy streams of the library's own, so step n+1's uploads and step n's downloads overlap
 * step n's compute:
 *   atjup_gpu_upload_async(ctx, id, host)    queue the copy of host (contiguous (i, j, k), pinned
 *                                            for overlap) into a device staging buffer;
 *   atjup_gpu_apply_uploads(ctx)             make the fields queued since the last call live, in
 *                                            the order of the library's compute stream;
 *   atjup_gpu_download_async(ctx, id, host)  snapshot the field in the compute stream's order and
 *                                            queue its copy to host.
 * Host buffers must stay untouched until atjup_gpu_synchronize, which waits for the copy streams
 * too. A field takes effect only through atjup_gpu_apply_uploads; the time-level-n copies of the
 * scalars are not touched (as with atjup_gpu_upload). Staging: two device copies of each field
 * used, allocated on first use. */
int atjup_gpu_upload_async(AtjupCtx* ctx, int32_t field_id, const double* host);
int atjup_gpu_apply_uploads(AtjupCtx* ctx);
int atjup_gpu_download_async(AtjupCtx* ctx, int32_t field_id, double* host);

/* cJupiterModel::RungeKuttaJup (RungeKutta_Jup_Turb.cpp:261-583): buoyancy level mean,
 * hydrostatic pressure, four fused RK stages (RHSJup per cell, RHS_Jup_Turb.cpp:31-1457). */
int atjup_gpu_rk4_step(AtjupCtx* ctx, int32_t iter_n);
/* Stage buffers of the FP64 dry RK step: with bufs (12 device buffers in the padded layout,
 * stage-major X1 t, u, v, w, X2 .., X3 ..) every following RK step writes its stage inputs there
 * instead of the context's own buffers, so that they outlive the step as the adjoint's checkpoint
 * (atjup_gpu_iteration_adjoint_ckpt); NULL returns to the context's buffers. No counterpart in the
 * reference. Each buffer 16-byte aligned (ATJUP_ERR_ARG otherwise: the stage kernel reads its
 * input through tensor maps). ATJUP_ERR_UNSUPPORTED with the physics block or the mixed step. */
int atjup_gpu_set_stage_buffers(AtjupCtx* ctx, double* const bufs[12]);

/* PressureSolverJup::run (PressureSolver.h:144-766) incl. prepareProjectionBoundaries
 * (cJupiterModel.cpp:1842-1864). SWEEPS reproduces the reference; RESIDUAL solves the same
 * operator to opts->rel_tol. stats may be NULL. */
int atjup_gpu_pressure_solve(AtjupCtx* ctx, const AtjupSolveOpts* opts, AtjupSolveStats* stats);

/* Right-hand side for an isolated solve (contiguous, i,j,k; interior rows are read). */
int atjup_gpu_set_solve_rhs(AtjupCtx* ctx, const double* host_b);

/* Boundary passes: BC_Jup::bcRadius, bcTheta, bcPhi, bcSolidGround (BC_Jup.h:185-658). */
enum { ATJUP_BC_RADIUS = 1, ATJUP_BC_THETA = 2, ATJUP_BC_PHI = 4, ATJUP_BC_SOLID = 8,
       ATJUP_BC_ALL = 15 };
int atjup_gpu_bc(AtjupCtx* ctx, int32_t which);

/* JupiterUtils::damp_wiggles (order 2) / damp_wiggles_ho (order 4), lib/Utils.cpp:227-453,
 * k then j then i passes, with i_topography as the fluid floor when use_topo. */
int atjup_gpu_shapiro(AtjupCtx* ctx, int32_t field_id, int32_t order, double strength,
                      int32_t passes, int32_t use_topo);

/* cJupiterModel::computeMixtureDensity (InitValues_Jup.cpp:717-740). */
int atjup_gpu_mixture_density(AtjupCtx* ctx);

/* cJupiterModel::balanceColumnV (InitValues_Jup.cpp:1500-1538); vshift may be NULL. */
int atjup_gpu_balance_column_v(AtjupCtx* ctx, double* vshift);

/* cJupiterModel::projectAroundObstacle(in_loop = true) (InitValues_Jup.cpp:1595-1822): per level
 * that cuts the obstacle, the divergence solve (cone_proj_div > 0) and the wall-flux solve, each
 * warm-started from its own phi of the previous call (zero before the first), v and w incremented,
 * then the seam copy of v and w. atjup_gpu_step calls it every cone_proj_stride iterations; this
 * entry runs one call on its own. The result is the reference's to the bit. */
int atjup_gpu_cone_project(AtjupCtx* ctx);
/* The levels of the projection and the SOR sweeps of its last call, per level: sweeps[2 l] of the
 * divergence solve (0 when off), sweeps[2 l + 1] of the wall-flux solve (40001: not converged
 * within 40000 sweeps, the reference's count). Fills up to cap levels; *n_levels = all levels. */
int atjup_gpu_cone_stats(AtjupCtx* ctx, int32_t* level_i, int32_t* sweeps, int32_t cap,
                         int32_t* n_levels);

/* The column balance of v for callers that cannot allocate device memory. No counterpart in the
 * reference: it computes what atjup_gpu_balance_column_v computes, on the caller's own device
 * buffers -- v (in/out, [im][jm][pitch] doubles), i_topo ([jm * km] int32), rad ([im]) -- and keeps
 * its scratch in a fixed file-scope device array instead of allocating. For host models that hand
 * the GPU layer one memory pool sized at start-up and allow no allocation after it, and for
 * embeddings that must not fail part-way through a run on an out-of-memory allocation.
 * Limits: jm <= ATJUP_NOALLOC_MAX_J, pitch <= ATJUP_NOALLOC_MAX_PITCH, else ATJUP_ERR_ARG. The
 * first call on each device looks up the array's device address (cudaGetSymbolAddress) and keeps
 * it for the life of the process; make that first call before any stream capture. The kept
 * address does not survive cudaDeviceReset: after a reset, do not call this entry point again in
 * the same process. Calls share the array: calls that overlap on the GPU race.
 * stream: a cudaStream_t or NULL. */
#define ATJUP_NOALLOC_MAX_J 256
#define ATJUP_NOALLOC_MAX_PITCH 512
int atjup_gpu_balance_column_v_noalloc(double* v, const int32_t* i_topo, const double* rad,
                                       int32_t im, int32_t jm, int32_t km, int32_t pitch,
                                       double dr, int32_t zonal, void* stream);

/* ---- full physics in the RK4 step (RHS_Jup_Turb.cpp:132-303, 459-998, 1266-1452) ---- */

/* The transported scalars, in the order RHSJup writes them (RHS_Jup_Turb.cpp:1273-1333). */
enum { ATJUP_S_H2O = 0, ATJUP_S_H2O_CLOUD, ATJUP_S_H2O_ICE, ATJUP_S_H2S, ATJUP_S_NH3,
       ATJUP_S_NH3_CLOUD, ATJUP_S_NH3_ICE, ATJUP_S_CH4, ATJUP_S_CH4_CLOUD, ATJUP_S_CH4_ICE,
       ATJUP_S_NH4SH, ATJUP_S_COUNT };
enum { ATJUP_TURB_K_EPSILON = 0, ATJUP_TURB_K_OMEGA = 1, ATJUP_TURB_K_OMEGA_SST = 2 };

typedef struct AtjupPhysics {
    int32_t species_on;          /* 1: the 11 species are integrated with the dynamics           */
    int32_t turb_on;             /* use_turbulence_model (ATJUP_TURB, turb_model; default on)     */
    int32_t turb_model;          /* ATJUP_TURB_MODEL / turb_model, default k_omega_SST            */
    int32_t turb_buoy;           /* ATJUP_TURB_BUOY 0: buoyancy production of k* (RHS:963-981)   */
    double species_diff_scale;   /* ATJUP_SPECIES_DIFF_SCALE 0.01 (cJupiterModel.h:470)          */
    double sc_h2o, sc_h2s, sc_nh3, sc_ch4, sc_nh4sh;   /* Schmidt numbers (cJupiterModel.h:473) */
    double chemical_reaction;    /* coupling of the chemistry mass fluxes                        */
    double r_p_nh4sh, rg_nh4sh;  /* NH4SH crystal radius [m] and density [kg/m3] (Stokes fall)   */
    double mue_mix;              /* dynamic viscosity of the mixture                              */
    double re_turb;              /* k-epsilon near-wall term scale (TurbulenceJup)                */
    double nue_max_phys;         /* ATJUP_NUE_MAX 1e5 m2/s (Turbulence.h:123)                     */
    double tke_max_phys;         /* ATJUP_TKE_MAX 1000 m2/s2 (RungeKutta_Jup_Turb.cpp:269)        */
    double turb_buoy_prt;        /* ATJUP_TURB_BUOY_PRT 0.9                                       */
    /* the closure update between steps (Turbulence.h:307-882, atjup_gpu_turbulence)              */
    int32_t turb_free;           /* ATJUP_TURB_FREE 1: no surface law, u_tau = 0.05 m/s           */
    int32_t turb_curv;           /* ATJUP_TURB_CURV 1: curvature terms of the velocity gradient   */
    int32_t abl_taper;           /* ATJUP_ABL_TAPER 0: taper nue above the boundary layer         */
    int32_t turb_wall_omega;     /* ATJUP_TURB_WALL_OMEGA 1 (cJupiterModel.cpp:360-377)           */
    double turb_k_bg;            /* ATJUP_TURB_K_BG 1 m2/s2: background k floor (TURB_FREE)       */
    double vel_star_max;         /* ATJUP_VEL_STAR_MAX sqrt(0.002) 200 m/s                        */
    double abl_height;           /* abl_height 20000 m (cJupiterModel.h:1534)                     */
} AtjupPhysics;

/* Switch the RK4 step to full physics: the 11 species and (turb_on) k*, omega* are integrated
 * with t, u, v, w, each with its own time-level-n copy (the reference's h2on .. disn).
 * layer_heights_km[im] is m_layer_heights (float, km), the wall distance of the closure.
 * Allocates the scalar stage buffers on first use. phys = NULL switches back to dynamics only. */
int atjup_gpu_set_physics(AtjupCtx* ctx, const AtjupPhysics* phys, const float* layer_heights_km);
/* Switch the precision of the RK step (AtjupParams.precision) between steps. No reference
 * counterpart: the reference computes in FP64 only. */
int atjup_gpu_set_precision(AtjupCtx* ctx, int32_t precision);
/* The time-level-n copy of a transported scalar (field ids ATJUP_F_H2O .. ATJUP_F_DIS). */
int atjup_gpu_upload_n(AtjupCtx* ctx, int32_t field_id, const double* host);
int atjup_gpu_download_n(AtjupCtx* ctx, int32_t field_id, double* host);
/* restoreVar for the scalars (cJupiterModel.cpp:1757-1801): n copy <- live field. */
int atjup_gpu_restore_scalars(AtjupCtx* ctx);
/* Turbulence<cJupiterModel>::run (Turbulence.h:307-328: friction velocity, production and
 * sources with the two clamp passes, wall law, obstacle zeroing, nue clamp, seam and lid copies)
 * followed by the driver's turbWallOmega (cJupiterModel.cpp:360-377). Updates tke, dis, their
 * time-level-n copies where the reference does, nue, prod, tke_source, dis_source, vel_star. */
int atjup_gpu_turbulence(AtjupCtx* ctx);
/* 2-D fields, contiguous (j, k). */
int atjup_gpu_upload2d(AtjupCtx* ctx, int32_t field_id, const double* host);
int atjup_gpu_download2d(AtjupCtx* ctx, int32_t field_id, double* host);

/* ---- saturation adjustment (SaturationAdjustment.h:255-746, Tao et al. 1988) ---- */
enum { ATJUP_GAS_H2O = 0, ATJUP_GAS_NH3 = 1, ATJUP_GAS_CH4 = 2 };

/* One gas: the 14 constants cJupiterModel passes to SaturationAdjustmentJup::run
 * (SaturationAdjustment.h:236-243, cJupiterModel.cpp:1060-1080) and the knobs the routine reads
 * once per planet (ATJUP_SATADJ_*, SaturationAdjustment.h:277-307; defaults cJupiterModel.h:
 * 1045-1057). The saturation vapour pressure is exp(C + (-L0/T + del_alf ln T + del_bet T) /
 * (1e-3 R)) [bar] (ATPhys.h:49-52); the *_i set is the ice one. */
typedef struct AtjupGasParams {
    double t_0, t_00;            /* all-liquid above t_0, all-ice below t_00 [K]                 */
    double ep, lv, ls;           /* molar-mass ratio, latent heats of vaporisation / sublimation */
    double C, L0, R, del_alf, del_bet;          /* liquid vapour-pressure set, R [J/(kg K)]     */
    double C_i, L0_i, del_alf_i, del_bet_i;     /* ice vapour-pressure set                      */
    int32_t conserve;            /* ATJUP_SATADJ_CONSERVE 1: melt (not delete) ice above t_0     */
    int32_t newton;              /* ATJUP_SATADJ_NEWTON 1: damped Newton step of the target      */
    int32_t evap;                /* ATJUP_SATADJ_EVAP 1: cells with condensate off target enter  */
    int32_t ice_entry;           /* ATJUP_SATADJ_ICE_ENTRY 0: temperature-split entry target     */
    int32_t bergeron;            /* ATJUP_SATADJ_BERGERON 2                                      */
    int32_t freeze;              /* ATJUP_SATADJ_FREEZE 0: liquid below t_00 freezes             */
    int32_t dry_exit;            /* ATJUP_SATADJ_DRY_EXIT 1: stop a dry, subsaturated cell       */
    int32_t reserved;
} AtjupGasParams;

typedef struct AtjupSatStats {
    int64_t adjusted;            /* cells that entered the mixed-phase iteration                 */
    int64_t not_converged;       /* of those, cells that used all 15 passes                      */
    int64_t dry_exits;           /* of those, cells that left through the dry exit               */
} AtjupSatStats;

/* SaturationAdjustmentJup(*this).run(gas, ...) on the device fields of one gas (vapour, cloud,
 * ice: ATJUP_F_H2O.. / NH3.. / CH4..), with t, p_stat, rho_mix (ATJUP_LOCAL_RHO) and the solid
 * mask; updates t and the three species in place. stats may be NULL. */
int atjup_gpu_satadj(AtjupCtx* ctx, int32_t gas, const AtjupGasParams* gp, AtjupSatStats* stats);

/* ---- the loop's microphysics (Radiation.h, Precipitation.h, ChemistryJup.h) ---- */

/* Every constant and knob of the moist part of the iteration, resolved on the host. */
typedef struct AtjupMicro {
    int32_t radiation_on;        /* ATJUP_RADIATION 1                                             */
    int32_t precip_on;           /* ATJUP_PRECIP 1                                                */
    int32_t nh4sh_eq;            /* ATJUP_NH4SH_EQ 1: NH4SH by equilibrium (ChemistryJup.h:285);  */
                                 /* 0: by the reaction-rate law (ChemistryJup.h:135-235)          */
    int32_t satadj_on;           /* the three gas adjustments (always on in the reference)        */
    int32_t solar_on;            /* ATJUP_SOLAR 1                                                 */
    int32_t rad_bottom;          /* ATJUP_RAD_BOTTOM 0: lower boundary of the thermal stream      */
    int32_t precip_coupling_on;  /* ATJUP_PRECIP_COUPLING != 0: sources, not in-place removal     */
    int32_t diagnostics_on;      /* 1: Forces and Latent_Heat close the physics block, as in the  */
                                 /* loop (cJupiterModel.cpp:1163-1164)                             */
    int32_t costhe_abs;          /* ATJUP_COSTHE_ABS 0 (cJupiterModel.h:1131-1134)                 */
    int32_t qheat_scale;         /* ATJUP_QHEAT_SCALE 0 (cJupiterModel.h:963-970)                  */
    int32_t pad;
    /* radiation (Radiation.h:166-487, cJupiterModel.h:1109-1118)                                 */
    double F_int, S_solar, albedo_bond, x_H2, x_He;
    double cia_strength;         /* ATJUP_CIA_STRENGTH 3.9                                        */
    double opacity_strength;     /* ATJUP_OPACITY_STRENGTH 1                                      */
    double solar_strength;       /* ATJUP_SOLAR_STRENGTH 1                                        */
    double sw_tau_per_bar;       /* ATJUP_SW_TAU_PER_BAR 1                                        */
    /* precipitation (Precipitation.h:93-140)                                                     */
    double precip_rate_scale;    /* ATJUP_PRECIP_SCALE 1                                          */
    /* chemistry (ChemistryJup.h:283-543, FluxLimiter.h)                                          */
    double m_nh3, m_h2s, m_nh4sh;          /* molar masses [kg/kmol]                              */
    double D_nh3, D_h2s, D_nh4sh;          /* mue / (rg sc): diffusivities of the mass fluxes     */
    double polar_divisor_floor;            /* 0.4 (ATPhys.h:104-108)                              */
    double t_0_nh4sh, t_00_nh4sh;          /* 230, 200 K: the rate law's NH4SH formation window   */
                                           /* (cJupiterModel.h:194-195; nh4sh_eq = 0)             */
    double cc[8];                          /* Latent_Heat's Clausius-Clapeyron E = exp(A/T + B):  */
                                           /* A, B, A_i, B_i of H2O, then of NH3                  */
                                           /* (cJupiterModel.h:222-240)                            */
    AtjupGasParams gas[3];                 /* H2O, NH3, CH4                                        */
} AtjupMicro;

/* Set (or with NULL clear) the microphysics of the iteration; with it and the physics block set,
 * atjup_gpu_step runs the full-physics schedule of the loop. */
int atjup_gpu_set_micro(AtjupCtx* ctx, const AtjupMicro* micro);
/* cJupiterModel::Forces (InitValues_Jup.cpp:742-812) and Latent_Heat (Thermo_Jup.cpp:89-232):
 * the Coriolis, centrifugal, buoyancy and pressure-gradient force densities and the latent and
 * sensible heating, output fields that nothing in the step reads. atjup_gpu_step runs it at the
 * end of the physics block when AtjupMicro.diagnostics_on is set. */
int atjup_gpu_diagnostics(AtjupCtx* ctx);
/* Radiation<cJupiterModel>::run (Radiation.h:251-487): grey two-stream fluxes per column -> Q_rad. */
int atjup_gpu_radiation(AtjupCtx* ctx);
/* Precipitation<cJupiterModel>::run (Precipitation.h:191-445): the three-category column scheme of
 * H2O, NH3, CH4 -> S_precip_* and Q_precip (or in-place removal when the coupling is off). */
int atjup_gpu_precipitation(AtjupCtx* ctx);
/* ChemistryJup::EquilibriumNH4SH("loop") (ChemistryJup.h:291-373): the NH4SH / NH3 + H2S
 * equilibrium per cell by bisection, with its latent heat. */
int atjup_gpu_nh4sh_equilibrium(AtjupCtx* ctx);
/* The chemistry block of the loop: DiffMassFluxJup's diffusive fluxes (ChemistryJup.h:375-538),
 * their 1-2-1 smoothing, ChemMassRateJup (59-281; massflux = reaction rate + difflux, the rate
 * zero with the equilibrium on),
 * FluxLimiterNH4SH (FluxLimiter.h) and the smoothing of the mass fluxes (cJupiterModel.cpp:
 * 1144-1162). */
int atjup_gpu_chemistry(AtjupCtx* ctx);
/* cJupiterModel::clampNegativeSpecies (FileIO_Jup.cpp:494-548): species < 0 or NaN -> 0. */
int atjup_gpu_clamp_species(AtjupCtx* ctx);

/* ---- moist convective adjustment, Ledoux criterion (ConvectiveAdjustment.h:275-849) ---- */

/* The knobs of MoistConvectiveAdjustment<cJupiterModel>::run (ConvectiveAdjustment.h:403-420) and
 * the driver's tracer constants (cJupiterModel.cpp:1300-1320). The two gases are H2O and NH3 with
 * the saturation constants of the micro block (AtjupMicro.gas[0], gas[1]); the tracers are H2S (a
 * gas in the virtual temperature, ep_h2s) and NH4SH (a condensate carrying its heat of formation,
 * L_nh4sh). The reference's chromophore tracer is zero unless ATJUP_CHROM is on, which this
 * library does not provide. Latitude smoothing (MCA_SMOOTH > 0), the temperature-split phase rule
 * (MCA_PHASE 1) and cp(T) (CP_H2, CP_GAS) are Jupiter's defaults off and not provided. */
typedef struct AtjupMca {
    int32_t stride;              /* ATJUP_MCA 1: every N iterations, after the boundary passes   */
    int32_t ledoux;              /* ATJUP_MCA_LEDOUX 1: composition in the density test          */
    int32_t loading;             /* ATJUP_MCA_LOADING 1: condensate weight in the density test   */
    int32_t interior;            /* ATJUP_MCA_INTERIOR 1: radial boundary planes left out        */
    int32_t max_pass;            /* ATJUP_MCA_PASSES 64: sweep cap per column                    */
    int32_t pad;
    double relax;                /* ATJUP_MCA_RELAX 1: fraction of the adjustment applied        */
    double ep_h2s;               /* 15.35: H2S molar-mass ratio (cJupiterModel.h:418)            */
    double L_nh4sh;              /* NH4SH heat of formation [J/kg] with ATJUP_NH4SH_EQ, else 0   */
} AtjupMca;

typedef struct AtjupMcaStats {
    int64_t columns;             /* columns adjusted                                             */
    int64_t layers;              /* cells mixed, summed over the segments                        */
    int64_t moist_triggers, dry_triggers;   /* first-sweep segments started by a saturated /    */
                                            /* unsaturated parcel                               */
    int64_t unstable_t, held;    /* pairs unstable in T; of those, held by their composition    */
    int64_t skipped;             /* columns left alone (no positive state, failed solve)         */
    int32_t max_passes, pad;     /* the most sweeps a column used                                */
} AtjupMcaStats;

/* Set (or with NULL clear) the moist convective adjustment of the iteration; needs the micro
 * block (the gases' constants) and the physics block (the species). */
int atjup_gpu_set_mca(AtjupCtx* ctx, const AtjupMca* mca);
/* MoistConvectiveAdjustment<cJupiterModel>::run on the device state: t and the H2O, NH3, H2S,
 * NH4SH fields of every column that holds an unstable pair. stats may be NULL. */
int atjup_gpu_mca(AtjupCtx* ctx, AtjupMcaStats* stats);

/* One iteration of cJupiterModel::Run's loop (cJupiterModel.cpp:1032-1381). Dry: pressure
 * solve on even iterations (and when first != 0), mixture density, RK4, boundary passes,
 * in-loop Shapiro, column balance of v; restoreVar is implicit (the device state is the time
 * level n copy). With atjup_gpu_set_physics and atjup_gpu_set_micro set, the full-physics
 * schedule: on even iterations (and the first) also radiation, the H2O, NH3, CH4 saturation
 * adjustments, the NH4SH equilibrium, precipitation, the n copies of the condensables, the
 * turbulence update and the chemistry block; every iteration RK4 of the 17 fields, the boundary
 * passes of every field list, the closure's wall hold, the moist convective adjustment (when set,
 * on its stride), Shapiro, the column balance, the species clamp and restoreVar of the scalars. solve may be NULL (= params->press_sweeps sweeps). */
int atjup_gpu_step(AtjupCtx* ctx, int32_t iter_n, int32_t first, const AtjupSolveOpts* solve);

/* Count of non-finite values in the prognostic fields (NaN/Inf census; no device trap). */
int atjup_gpu_nonfinite_count(AtjupCtx* ctx, int64_t* count);

/* ---- restart files (FileIO_Jup.cpp:261-683) ---- */

/* cJupiterModel::save_state (FileIO_Jup.cpp:584-624): write the device state to `path` in the
 * reference's restart format -- header {magic, im, jm, km, iter} (int32), then every array of
 * restart_arrays() as im*jm rows of km doubles, and with carried != 0 (magic "JUP2") the arrays
 * of restart_arrays_carried() and vel_star, else magic "JUP1". Call it between steps (after
 * atjup_gpu_step), where every time-level-n copy equals its live field, as the reference does
 * after restoreVar. thermalmassflux, a diagnostic this library does not compute, is written as
 * zeros. carried = 2 also appends, after vel_star, a trailer ("ATJX", count, arrays) with the NH4SH
 * mass flux and the NH3-cloud and CH4 precipitation sinks, which the next iterations read but the
 * reference's list omits; the reference's loader does not read past vel_star. The reference names
 * the file <output_path>/jup_restart_<iter>.bin. */
int atjup_gpu_save_state(AtjupCtx* ctx, const char* path, int32_t iter, int32_t carried);
/* cJupiterModel::load_state (FileIO_Jup.cpp:626-683): read a JUP1 or JUP2 file written by the
 * reference or by atjup_gpu_save_state into the device state. The magic, the grid and the file
 * size are checked before any device field is written (ATJUP_ERR_ARG and a message otherwise).
 * iter receives the header's iteration, carried 0 for JUP1, 1 for JUP2, 2 for JUP2 with the
 * trailer of atjup_gpu_save_state. Resume with
 * atjup_gpu_step(iter + 1, first = !carried): the reference forces the physics block on the
 * first resumed iteration only for a JUP1 file. */
int atjup_gpu_load_state(AtjupCtx* ctx, const char* path, int32_t* iter, int32_t* carried);

/* Tangent-linear and adjoint of one RK4 step of the dry dynamics: RungeKuttaJup
 * (RungeKutta_Jup_Turb.cpp:261-583) with the t, u, v, w right-hand sides of RHSJup
 * (RHS_Jup_Turb.cpp:31-1457), the buoyancy level mean (47-69) and the hydrostatic integral
 * (119-259), linearised about the context's current t, u, v, w. p_dyn, p_stat, rho_mix, wall_nue
 * and the cell-hold means are inputs of the step and held fixed; the state is not advanced.
 * d / a are four device buffers (t, u, v, w) in the context's padded layout (atjup_gpu_field_ptr
 * gives the row pitch; lanes k >= km are ignored):
 *   atjup_gpu_rk4_tlm      d in: a perturbation of the time-level-n state; out: the step's
 *                          response (lanes k >= km set to 0)
 *   atjup_gpu_rk4_adjoint  a in: the adjoint of the step's result; out: of its input
 * Dry dynamics in FP64 only (ATJUP_ERR_UNSUPPORTED with the physics block, nue or heating on, or
 * the mixed step). The adjoint adds with FP64 atomics, so its last bits depend on their order.
 * (The reference has no derivative code.) */
int atjup_gpu_rk4_tlm(AtjupCtx* ctx, double* const d[4]);
int atjup_gpu_rk4_adjoint(AtjupCtx* ctx, double* const a[4]);

/* Tangent-linear and adjoint of one whole dry iteration of cJupiterModel::Run's loop
 * (cJupiterModel.cpp:1032-1381 with the dry knobs): on even iterations (and when first != 0) the
 * pressure pass (PressureSolver.h:144-766, prepareProjectionBoundaries cJupiterModel.cpp:
 * 1842-1864; ATJUP_SOLVE_SWEEPS with press_sweeps sweeps, omega 1) and the mixture density
 * (InitValues_Jup.cpp:717-740); every iteration RungeKuttaJup, the boundary passes
 * (BC_Jup.h:185-658), the in-loop 4th-order Shapiro filter of u, v, w (lib/Utils.cpp:334-453)
 * and the column balance of v (InitValues_Jup.cpp:1500-1538). The linear state is nine device
 * buffers in the context's padded layout: t, u, v, w, p_dyn, aux_u, aux_v, aux_w, rho_mix (what
 * an iteration reads from the one before). Both linearise about the context's current state,
 * taken as the iteration's input, and leave that state as they found it. The source clamp of the
 * pressure pass is linearised as its derivative at the base state (the perturbation passes where
 * the base divergence is not clamped).
 *   atjup_gpu_iteration_tlm      d in: a perturbation of the iteration's input; out: its response
 *   atjup_gpu_iteration_adjoint  a in: the adjoint of the iteration's output; out: of its input
 * parts selects the passes in the linear map (ATJUP_LIN_ALL: the whole iteration; a pass left out
 * is the identity), for checking them one at a time. Dry dynamics in FP64 only, as
 * atjup_gpu_rk4_tlm; an iteration at which the projection around the obstacle runs
 * (cone_proj_stride) is refused with ATJUP_ERR_UNSUPPORTED. (The reference has no derivative
 * code.) */
enum { ATJUP_LIN_PRESSURE = 1, ATJUP_LIN_MIXTURE = 2, ATJUP_LIN_RK4 = 4, ATJUP_LIN_BC = 8,
       ATJUP_LIN_SHAPIRO = 16, ATJUP_LIN_BALANCE = 32, ATJUP_LIN_ALL = 63 };
int atjup_gpu_iteration_tlm(AtjupCtx* ctx, int32_t iter_n, int32_t first, int32_t parts,
                            double* const d[9]);
int atjup_gpu_iteration_adjoint(AtjupCtx* ctx, int32_t iter_n, int32_t first, int32_t parts,
                                double* const a[9]);
/* The same with the RK step's stage inputs X1, X2, X3 of t, u, v, w (12 device buffers in the
 * padded layout, stage-major: X1 t, u, v, w, X2 .., X3 ..) kept by the forward iteration
 * (atjup_gpu_set_stage_buffers) instead of recomputed: a checkpoint of 12 fields per iteration
 * that saves three RK stages per adjoint iteration. */
int atjup_gpu_iteration_adjoint_ckpt(AtjupCtx* ctx, int32_t iter_n, int32_t first, int32_t parts,
                                     double* const a[9], const double* const stages[12]);
/* Device-to-device copy between a field and a caller's device buffer in the padded layout
 * (im * jm * pitch doubles), in the context's stream order: to_field 1 copies buf into the field,
 * 0 the field into buf. For callers that hold the state in their own device tensors (the torch
 * binding of the RK4 step). (No reference counterpart.) */
int atjup_gpu_copy_field(AtjupCtx* ctx, int32_t field_id, double* buf, int32_t to_field);

/* Instrumentation (no reference counterpart: the reference prints wall-clock timers per routine,
 * e.g. RungeKutta_Jup_Turb.cpp:577-579). With timing on, the library records a CUDA event pair
 * on its stream around every kernel launch of a class; atjup_gpu_timing_read sums them. Launches
 * that run on the library's second stream (the scalar RK stages, coupled precipitation, the moist
 * convective adjustment) are timed on it, so their times include the share of the GPU that the
 * concurrent work on the other stream takes. ATJUP_TK_RK_GROUP is one RK stage as a whole (the
 * scalar and dynamics kernels together), read from those events' first start and last end. */
enum { ATJUP_TK_RK_STAGE = 0, ATJUP_TK_RK_AUX, ATJUP_TK_PRESSURE, ATJUP_TK_BC, ATJUP_TK_SHAPIRO,
       ATJUP_TK_BALANCE_V, ATJUP_TK_MIXTURE, ATJUP_TK_SOLVER, ATJUP_TK_SATADJ, ATJUP_TK_SPECIES,
       ATJUP_TK_CLOSURE, ATJUP_TK_TURB, ATJUP_TK_MICRO, ATJUP_TK_MCA, ATJUP_TK_RK_GROUP,
       ATJUP_TK_CONE, ATJUP_TK_COUNT };
int atjup_gpu_timing(AtjupCtx* ctx, int32_t enable);   /* 1: reset and record; 0: stop */
int atjup_gpu_timing_read(AtjupCtx* ctx, int32_t kernel_class, double* total_ms, int64_t* count);
/* Number of kernels this context has launched since creation. */
int atjup_gpu_launch_count(AtjupCtx* ctx, int64_t* launches);

int atjup_gpu_synchronize(AtjupCtx* ctx);
const char* atjup_gpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* ATJUP_GPU_H */
