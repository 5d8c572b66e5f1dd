// Device context and shared helpers of the ATJUP B200 hot path.
//
// HBM layout: every 3-D field is a structure-of-arrays block [i][j][KP] of doubles with the
// longitude index k fastest and rows padded from km = 361 to KP = 368 elements, so each
// (i, j) row starts on a 128-byte boundary (368 * 8 = 23 * 128). Cell (i, j, k) lives at
// (i * jm + j) * KP + k. Padding elements are never read as data.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/atjup_gpu.h"

#define ATJUP_MAX_SOLVE_PARTIALS 1024

namespace atjup {

// Per-(i, j) geometry, computed on the host in double with the same expressions as the
// reference's CellGeometry (RungeKutta_Jup_Turb.cpp:388-411) and uploaded once.
struct GeoIJ {
    double rm, inv_rm, inv_rm2, inv_rmsinthe;
    double inv_rm2sinthe, inv_rm2sinthe2, costhe_inv_rm2sinthe, v_metric;
    double cotanthe, costhe, sinthe_true, cent_rad;
    double cent_the, cor_rad, cor_the, num2;   // cor_*: (nd_cor * -2 * omega) * sine / cosine
    double num3, pad0, pad1, pad2;             // num2 / num3: Poisson face weights of the row
};

// One solid cell of the obstacle with its bcSolidGround treatment (BC_Jup.h:496-590), found
// once from the static mask: a/b are the two fluid cells of the extrapolation (kind 1), or
// kind 0 (interior or no pair: p_dyn = 0).
struct SolidCell {
    int64_t c, a, b;
    int32_t kind, pad;
};

struct AtjupCtxImpl;

}  // namespace atjup

struct AtjupCtx {
    AtjupParams P;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // asynchronous field exchange (xfer.cu): copy streams, double-buffered staging by round
    bool xfer_on = false;
    cudaStream_t x_h2d = nullptr, x_d2h = nullptr;
    double* x_up[2][ATJUP_F_COUNT] = {};
    double* x_out[2][ATJUP_F_COUNT] = {};
    cudaEvent_t x_up_done[2] = {}, x_up_free[2][ATJUP_F_COUNT] = {}, x_out_free[2][ATJUP_F_COUNT] = {};
    cudaEvent_t x_out_ready = nullptr;
    unsigned long long x_pending[2] = {0, 0};
    long long x_round = 0;
    // a second compute stream: the species and closure kernels of an RK stage run on it beside
    // the dynamics kernel of the same stage (one fork and one join per stage)
    cudaStream_t side = nullptr;
    cudaEvent_t side_fork = nullptr, side_join = nullptr;
    int KP = 0;              // padded row pitch (elements)
    size_t NP = 0;           // im * jm * KP
    bool grid_set = false;

    // state and inputs (FP64); index by ATJUP_F_*
    double* f[ATJUP_F_COUNT] = {};
    double* f2[ATJUP_F2_COUNT] = {};   // 2-D fields [jm][KP]
    // full physics (atjup_gpu_set_physics): time-level-n copies of the transported scalars
    // (indexed by field id, allocated for the scalars only), their stage buffers and
    // accumulators (indexed ATJUP_S_*, then k*, omega*), the closure's layer heights
    bool phys_on = false;
    AtjupPhysics phys{};
    double* fn[ATJUP_F_COUNT] = {};
    double* S1[ATJUP_S_COUNT + 2] = {};
    double* S2[ATJUP_S_COUNT + 2] = {};
    double* Sacc[ATJUP_S_COUNT + 2] = {};
    float* layer_h = nullptr;
    double turb_taper_dz = 1.0;        // clamp_nue's taper depth (Turbulence.h:569-573) [m]
    // the loop's microphysics (atjup_gpu_set_micro)
    bool micro_on = false;
    // storage of the RK stage buffers and accumulators: ATJUP_PREC_FP64, or ATJUP_PREC_MIXED (FP32)
    int step_prec = ATJUP_PREC_FP64;
    AtjupMicro micro{};
    // moist convective adjustment (mca.cu)
    bool mca_on = false;
    AtjupMca mca{};
    void* mca_bounds = nullptr;     // int2 [jm * km]: the column's (i0, i1)
    void* mca_flags = nullptr;      // unsigned [2 * jm * km + 1]: flags, list, count
    void* mca_slots = nullptr;      // per-thread column scratch of the column kernel
    void* mca_pairs = nullptr;      // uint8 [im * jm * km]: the census result of every pair
    void* mca_stats = nullptr;      // unsigned long long [8 + 2 * partials]
    double* cos_lat = nullptr;         // [jm] max(0, sin(pi j / (jm - 1))), the solar geometry
    // RK stage buffers and accumulators for t, u, v, w
    double* X1[4] = {};
    double* X2[4] = {};
    // caller buffers for the stage inputs X1, X2, X3 of t, u, v, w (atjup_gpu_set_stage_buffers):
    // the FP64 dry step writes its stages there, where an adjoint can take them as checkpoints
    double* keep[12] = {};
    bool keep_on = false;
    double* acc[4] = {};
    // scratch
    double* src = nullptr;       // Poisson source, one value per cell
    double* tmp = nullptr;       // filter ping-pong buffers
    double* tmp2 = nullptr;
    double* stage = nullptr;     // contiguous (unpadded) transfer buffer, im*jm*km doubles
    double* red = nullptr;       // reduction partials
    double* buoy_ref = nullptr;  // [im]
    double* zm = nullptr;        // [4 * jm] zonal means for the top sponge
    double* dvc = nullptr;       // [jm * KP] column means of v
    double* dvrow = nullptr;     // [jm]
    // Krylov solver vectors (allocated on first RESIDUAL solve)
    double* kr[8] = {};
    float* kf[8] = {};
    double* solve_b = nullptr;   // external right-hand side
    double* dsum = nullptr;      // [ATJUP_MAX_SOLVE_PARTIALS * 4] dot-product partials
    double* hsum = nullptr;      // pinned host copy of the final dot products
    unsigned long long* counters = nullptr;  // [8] event counters of the last satadj call
    double* lin = nullptr;       // scratch of the RK4 tangent-linear / adjoint (adjoint.cu)
    double* itlin = nullptr;     // scratch of the iteration's tangent-linear / adjoint (iteration_lin.cu)

    // static grid
    uint8_t* solid = nullptr;
    uint8_t* nbflags = nullptr;    // per-cell neighbour-solid and integrated flags (rk4.cu)
    int32_t* topo = nullptr;
    atjup::GeoIJ* geo = nullptr;   // [im * jm]
    double* cor_col = nullptr;     // [jm] Coriolis factor of the hydrostatic integral
    double* sin_the = nullptr;     // [jm] sin(the_j), the area weight of the level mean
    double* rad = nullptr;         // [im]
    double* cell_vbar0 = nullptr;  // [im * jm]
    double* cell_ubar0 = nullptr;
    atjup::SolidCell* solid_list = nullptr;
    int n_solid = 0;
    int32_t* amb_rows = nullptr;   // (i, j) rows that contain solid cells
    int n_amb_rows = 0;
    double* yw = nullptr;          // [NP] left null vector weight a_i d_j on fluid unknowns
    double* line_a = nullptr;      // radial line factors for the preconditioner
    double* line_c = nullptr;
    double* line_m = nullptr;
    double yw_sum = 0.0;
    void* solver = nullptr;           // residual-solver state (solver.cu), built on first use
    void* cone = nullptr;             // projection around the obstacle (cone.cu), built on first use

    // instrumentation: kernel launches issued, and CUDA-event timing per kernel class
    long long launches = 0;
    bool timing = false;
    std::vector<cudaEvent_t> tev;     // event pool, two per timed launch
    std::vector<int> tcls;            // class of each timed launch
    // the RK stages run on two streams: per stage the slot whose start opens it and the slots
    // whose ends close it (class TK_RK_GROUP is read from these, without events of its own)
    std::vector<int> tgrp;            // three slots per stage: start, end, end (-1: none)
    int tn = 0;                       // timed launches recorded
};

namespace atjup {

void set_error(const std::string& msg);

// kernel classes of the timing hook (atjup_gpu_timing)
enum { TK_RK_STAGE = 0, TK_RK_AUX, TK_PRESSURE, TK_BC, TK_SHAPIRO, TK_BALANCE_V, TK_MIXTURE,
       TK_SOLVER, TK_SATADJ, TK_SPECIES, TK_CLOSURE, TK_TURB, TK_MICRO, TK_MCA, TK_RK_GROUP,
       TK_CONE, TK_COUNT };
// an event pair per timed region: timer_begin records the start on st and returns the region's
// slot (-1 with timing off), timer_end records the end of that slot; regions may nest
int timer_begin(AtjupCtx* c, int cls, cudaStream_t st);
void timer_end(AtjupCtx* c, int slot, cudaStream_t st);
int cuda_status(cudaError_t e, const char* what);

inline size_t cell(const AtjupCtx* c, int i, int j, int k) {
    return ((size_t)i * c->P.jm + j) * c->KP + k;
}

// launchers (return ATJUP_OK or an error code)
int launch_buoy_ref(AtjupCtx* c, const double* t);
int launch_hydrostatic(AtjupCtx* c, const double* v, const double* w);
int launch_rk_stage(AtjupCtx* c, int stage, const void* const* Xin, void* const* Xout,
                    const void* const* X1);
int mca_setup(AtjupCtx* c);
int launch_mca(AtjupCtx* c);
int mca_read_stats(AtjupCtx* c, unsigned long long* out);
int launch_mixture_density(AtjupCtx* c);
int launch_prepare_projection(AtjupCtx* c);
int launch_pressure_source(AtjupCtx* c);
int launch_pressure_sweep(AtjupCtx* c, int colour, double omega);
int launch_prepare_projection_ptr(AtjupCtx* c, double* au, double* av, double* aw);
int launch_pressure_source_ptr(AtjupCtx* c, const double* au, const double* av, const double* aw,
                               double* src, const uint8_t* mask_in, uint8_t* mask_out);
int launch_pressure_sweep_ptr(AtjupCtx* c, double* p, const double* src, int colour, double omega);
int launch_pressure_fold(AtjupCtx* c, double* p);
int launch_bc(AtjupCtx* c, int which);
int launch_bc_ptrs(AtjupCtx* c, int which, double* t, double* u, double* v, double* w,
                   double* p_dyn, double* p_stat, bool phys);
int rk4_tlm_ext(AtjupCtx* c, double* const d[4], const double* dp, const double* drho,
                double* const daux[3]);
// stages: the forward's stage inputs X1, X2, X3 of t, u, v, w (12 buffers, stage-major), or null
// to recompute them
int rk4_adjoint_ext(AtjupCtx* c, double* const a[4], double* lp, double* lrho,
                    double* const laux[3], const double* const* stages = nullptr);
int launch_shapiro(AtjupCtx* c, double* f, int order, double strength, int passes, int use_topo);
int launch_balance_v(AtjupCtx* c);
int cone_prepare(AtjupCtx* c);
int launch_cone_projection(AtjupCtx* c);
void cone_free(AtjupCtx* c);
int launch_balance_v_buffers(double* v, const int32_t* topo, const double* rad, double* dvc,
                             double* dvrow, int im, int jm, int km, int pitch, double dr,
                             int zonal, cudaStream_t st);
int launch_nonfinite(AtjupCtx* c, unsigned long long* d_count);
int launch_pad(AtjupCtx* c, const double* flat, double* padded);     // (i,j,k) km -> KP rows
int launch_unpad(AtjupCtx* c, const double* padded, double* flat);
void xfer_free(AtjupCtx* c);
int xfer_synchronize(AtjupCtx* c);
int launch_satadj(AtjupCtx* c, int gas, const AtjupGasParams& gp);
extern const int kScalarField[ATJUP_S_COUNT + 2];
int launch_phys_stage(AtjupCtx* c, int stage, const void* const* vin, int what, cudaStream_t st);
int launch_turbulence(AtjupCtx* c);
int launch_turb_wall_hold(AtjupCtx* c);
enum { MICRO_RADIATION = 0, MICRO_PRECIP, MICRO_NH4SH, MICRO_CHEMISTRY, MICRO_CLAMP, MICRO_DIAG };
int launch_micro(AtjupCtx* c, int what);
int pressure_residual_solve(AtjupCtx* c, const AtjupSolveOpts* o, AtjupSolveStats* st);
void solver_free(AtjupCtx* c);

}  // namespace atjup

#define ATJUP_CUDA(call)                                                       \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) return atjup::cuda_status(e_, #call);           \
    } while (0)

#define ATJUP_CHECK_LAUNCH(what)                                               \
    do {                                                                       \
        cudaError_t e_ = cudaGetLastError();                                   \
        if (e_ != cudaSuccess) return atjup::cuda_status(e_, what);            \
    } while (0)
