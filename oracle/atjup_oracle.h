/*
 * CPU oracle for the ATJUP hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's time-step routines (RogerGrundmann/ATJUP), written
 * to check the CUDA implementation. Only tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg of bench.py load it; the product path never links or calls it.
 *
 * Parity pin: every routine here is compared, field by field, with the unmodified reference
 * built from its own sources (oracle/_ref/libatjup_ref.so via oracle/ref_harness.cpp) on the
 * reference's own initial state, and with the golden digests under tests/golden/ generated
 * from it (tests/golden/make_golden.py).
 *
 * Storage: contiguous (i, j, k) blocks, k fastest, idx = (i*jm + j)*km + k -- the same order as
 * the reference's x[i][j][k]. Any im, jm, km >= 5 works (the reference is fixed at 41x181x361;
 * small grids make fast GPU-vs-oracle tests).
 */
#ifndef ATJUP_ORACLE_H
#define ATJUP_ORACLE_H

#include <stdint.h>
#include "../include/atjup_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const double* rad;          /* [im] metric radius                                   */
    const double* the;          /* [jm] colatitude                                      */
    const uint8_t* solid;       /* [im*jm*km] SeaMount mask                             */
    const int32_t* topo;        /* [jm*km] i_topography                                 */
    const double* cell_vbar0;   /* [im*jm] or NULL                                      */
    const double* cell_ubar0;   /* [im*jm] or NULL                                      */
} ora_grid;

typedef struct {
    double *t, *u, *v, *w;              /* live fields (stage inputs inside the RK step)     */
    double *tn, *un, *vn, *wn;          /* time-level n copies                                */
    double *p_dyn, *p_hydro, *p_stat;
    double *rho_mix, *wall_nue, *nue;   /* nue may be NULL (closure off)                      */
    double *p_baro;                     /* may be NULL (no geo-balance rest)                  */
    double *aux_u, *aux_v, *aux_w;
    double *acc_t, *acc_u, *acc_v, *acc_w;
    double *rhs_t, *rhs_u, *rhs_v, *rhs_w;
    double *Q_rad, *Q_precip;           /* may be NULL (no heating)                           */
    double *buoy_ref;                   /* [im]                                               */
} ora_state;

/* The full-physics fields of the RK4 step: the 11 species in ATJUP_S_* order and k*, omega*
 * (live, time-level n, accumulator, right-hand side), their frozen sources, the closure's
 * outputs and inputs. */
typedef struct {
    double *q[ATJUP_S_COUNT], *qn[ATJUP_S_COUNT], *acc_q[ATJUP_S_COUNT], *rhs_q[ATJUP_S_COUNT];
    double *tke, *dis, *tken, *disn, *acc_tke, *acc_dis, *rhs_tke, *rhs_dis;
    const double* s_precip[9];   /* h2o, h2o_cloud, h2o_ice, nh3, .., ch4_ice                  */
    const double *massflux_h2s, *massflux_nh3, *massflux_nh4sh, *fluxlim_nh4sh;
    double *prod, *tke_source, *dis_source;
    double* vel_star;            /* [jm*km] friction velocity (written by ora_turbulence)      */
    double* nue_out;             /* the eddy viscosity ora_turbulence writes (the model's nue)  */
    const float* layer_heights;  /* [im] km                                                     */
    double* difflux[3];          /* diffusive fluxes of h2s, nh3, nh4sh (chemistry block)      */
} ora_phys;

/* RungeKutta_Jup_Turb.cpp:47-69 */
void ora_buoy_ref_level(const AtjupParams* P, const ora_grid* G, ora_state* S);
/* RungeKutta_Jup_Turb.cpp:119-259 (metric/Coriolis split branch and the plain branch) */
void ora_hydrostatic(const AtjupParams* P, const ora_grid* G, ora_state* S);
/* RHS_Jup_Turb.cpp:31-1457, dynamics part (t, u, v, w, aux) for one cell */
void ora_rhs_cell(const AtjupParams* P, const ora_grid* G, ora_state* S, int i, int j, int k);
/* RungeKutta_Jup_Turb.cpp:261-583 for t, u, v, w */
void ora_rk4(const AtjupParams* P, const ora_grid* G, ora_state* S);
/* RHS_Jup_Turb.cpp species and closure part for one cell (after ora_rhs_cell's dynamics) */
void ora_rhs_phys_cell(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G,
                       ora_state* S, ora_phys* X, int i, int j, int k);
/* RungeKutta_Jup_Turb.cpp:261-583 with the species and k*, omega* */
void ora_rk4_phys(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G, ora_state* S,
                  ora_phys* X);
/* Turbulence<cJupiterModel>::run (Turbulence.h:307-882) + turbWallOmega (cJupiterModel.cpp:
 * 360-377): reads u, v, w, t (S), tke/dis and their n copies, nue, vel_star (X); writes them. */
void ora_turbulence(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G, ora_state* S,
                    ora_phys* X);
/* cJupiterModel.cpp:1842-1864 */
void ora_prepare_projection(const AtjupParams* P, const ora_grid* G, ora_state* S);
/* PressureSolver.h:144-766, pointwise red-black branch, `sweeps` sweeps with relaxation omega
 * (omega = 1 is the reference). b != NULL replaces the divergence source by b (clamp skipped). */
void ora_pressure_sweeps(const AtjupParams* P, const ora_grid* G, ora_state* S, int sweeps,
                         double omega, const double* b);
/* The source the sweep uses at every interior cell (after the clamp) into src[N]. */
void ora_pressure_source(const AtjupParams* P, const ora_grid* G, ora_state* S, double* src);
/* A p for the folded-boundary operator the sweep relaxes (interior cells; 0 elsewhere). */
void ora_pressure_apply(const AtjupParams* P, const ora_grid* G, const double* p, double* Ap);
/* InitValues_Jup.cpp:717-740 */
void ora_mixture_density(const AtjupParams* P, const ora_grid* G, ora_state* S);
/* BC_Jup.h:185-263 + BoundaryConditions.h bcRadius/bcTheta/bcPhi; BC_Jup.h:460-658 */
void ora_bc_radius(const AtjupParams* P, const ora_grid* G, ora_state* S);
void ora_bc_theta(const AtjupParams* P, const ora_grid* G, ora_state* S);
void ora_bc_phi(const AtjupParams* P, const ora_grid* G, ora_state* S);
void ora_bc_solid(const AtjupParams* P, const ora_grid* G, ora_state* S);
/* the same passes over the full-physics field lists (X = NULL: the dynamics fields only) */
void ora_bc_radius_x(const AtjupParams* P, const ora_grid* G, ora_state* S, ora_phys* X);
void ora_bc_theta_x(const AtjupParams* P, const ora_grid* G, ora_state* S, ora_phys* X);
void ora_bc_phi_x(const AtjupParams* P, const ora_grid* G, ora_state* S, ora_phys* X);
void ora_bc_solid_x(const AtjupParams* P, const ora_grid* G, ora_state* S, ora_phys* X);
/* lib/Utils.cpp:227-323 (order 2) and 334-453 (order 4) */
void ora_shapiro(const AtjupParams* P, const ora_grid* G, double* f, int order, double strength,
                 int passes, int use_topo);
/* InitValues_Jup.cpp:1500-1538 */
double ora_balance_column_v(const AtjupParams* P, const ora_grid* G, ora_state* S);
/* InitValues_Jup.cpp:1595-1822 (projectAroundObstacle, in_loop = true): both solves per level
 * with warm starts phi_div / phi_wall ([im*jm*km], zero before the first call), v and w
 * incremented, the seam copied; sweeps ([2 * levels] or NULL) gets the SOR sweep counts
 * (0 for a solve that is off). Returns the number of levels. */
int ora_cone_project(const AtjupParams* P, const ora_grid* G, ora_state* S, double* phi_div,
                     double* phi_wall, int32_t* sweeps);
/* restoreVar (cJupiterModel.cpp:1757-1801) for the dynamics fields */
void ora_restore(const AtjupParams* P, ora_state* S);
/* SaturationAdjustment.h:255-746 for one gas (in place on t, c, cloud, ice); counts may be
 * NULL, else counts[0..2] = cells adjusted, not converged, dry exits. */
void ora_satadj(const AtjupParams* P, const ora_grid* G, const AtjupGasParams* g, double* t,
                const double* p_stat, const double* rho_mix, double* c, double* cloud,
                double* ice, long long* counts);
/* Radiation<cJupiterModel>::run (Radiation.h:251-487) -> S->Q_rad */
void ora_radiation(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G, ora_state* S,
                   ora_phys* X);
/* Precipitation<cJupiterModel>::run (Precipitation.h:191-445) -> S_precip_*, S->Q_precip */
void ora_precipitation(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G,
                       ora_state* S, ora_phys* X);
/* ChemistryJup::EquilibriumNH4SH("loop") (ChemistryJup.h:291-373) */
void ora_nh4sh_eq(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G, ora_state* S,
                  ora_phys* X);
/* The loop's chemistry block with the NH4SH equilibrium on: DiffMassFluxJup's difflux, 1-2-1
 * smoothing, ChemMassRateJup (massflux = difflux), FluxLimiterNH4SH, smoothing of the fluxes */
void ora_chemistry(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G, ora_state* S,
                   ora_phys* X);
/* clampNegativeSpecies (FileIO_Jup.cpp:494-548) */
void ora_clamp_species(const AtjupParams* P, ora_phys* X);
/* Turbulence.h:383-422 apply_wall_bc and the driver's turbWallOmega (cJupiterModel.cpp:360-377) */
void ora_turb_wall_bc(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G, ora_phys* X);
void ora_turb_wall_omega(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G, ora_phys* X);
/* MoistConvectiveAdjustment<cJupiterModel>::run (ConvectiveAdjustment.h:403-849); stats[8] */
void ora_mca(const AtjupParams* P, const AtjupMicro* MC, const AtjupMca* A, const ora_grid* G,
             ora_state* S, ora_phys* X, int64_t* stats);
/* One iteration of cJupiterModel.cpp:1032-1381 with the physics on; MCA may be NULL (off) */
void ora_iteration_phys(const AtjupParams* P, const AtjupPhysics* PH, const AtjupMicro* MC,
                        const AtjupMca* MCA, const ora_grid* G, ora_state* S, ora_phys* X,
                        int iter_n, int first, int sweeps);
/* One dry iteration of cJupiterModel.cpp:1032-1381 */
void ora_iteration_dry(const AtjupParams* P, const ora_grid* G, ora_state* S, int iter_n,
                       int first, int sweeps);

/* cJupiterModel::Forces (InitValues_Jup.cpp:742-812) and Latent_Heat (Thermo_Jup.cpp:89-232):
 * out = CoriolisForce, CentrifugalForce, BuoyancyForce, PresGradForce, Q_Latent, Q_Sensible */
void ora_diagnostics(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G,
                     const double* t, const double* u, const double* v, const double* w,
                     const double* p_dyn, const double* p_stat, const double* h2o,
                     const double* nh3, double* const* out);
size_t ora_micro_sizeof(void);

#ifdef __cplusplus
}
#endif
#endif
