// Full physics in the RK4 step: the 11 transported species and the k*, omega* pair of the
// turbulence closure, integrated stage by stage beside the dynamics (rk4.cu).
//
// Reference: RHS_Jup_Turb.cpp:132-303 (derivatives, with the solid-face mirror of k* and omega*),
// 482-545 (transport and diffusion), 736-998 (the closure's production and sources: k-epsilon,
// k-omega, k-omega SST, optional buoyancy production), 1266-1452 (the right-hand sides), and
// RungeKutta_Jup_Turb.cpp:419-568 (accumulation, next stage input, final assembly with the
// species floor at 0, the NaN-safe clamp of k* into [0, k_max], omega* >= 1e-10).
//
// A scalar's right-hand side needs its own 7-point stencil, the cell's velocities and nue, and
// its frozen sources, and no other scalar. So the species kernel is one thread per cell and
// species (k fastest, coalesced): it reads the stage input at the cell and its six neighbours (the
// k neighbours from the warp's own loads, the i and j neighbours mostly from L2), the
// time-level-n value and the accumulator, and writes the next stage input and the accumulator --
// 6 to 8 doubles of DRAM traffic per species per cell per stage. The closure kernel adds the nine velocity gradients its production
// term needs. Both kernels read the same stage input velocities as the dynamics kernel of the
// stage, and write only scalar buffers, so they are ordered freely against it.
//
// Non-integrated cells (the radial walls, three rows next to each pole, the seam copy, solid
// cells) keep their live values through the step: stages 0-2 copy the live field into the next
// stage input there, as the reference's untouched live arrays do.
#include "ctx.cuh"

namespace atjup {
namespace {

enum : uint8_t { NB_S = 1, NB_IP = 2, NB_IM = 4, NB_JP = 8, NB_JM = 16, NB_KP = 32, NB_KM = 64,
                 NB_INT = 128 };

struct PhysStage {
    // Stage buffers, typed by the kernel's template arguments: the stage input (velocities,
    // temperature, scalars), the next stage input (stage 3: the live field) and the accumulators.
    const void *u, *v, *w, *t;
    const void* q_in[ATJUP_S_COUNT + 2];
    void* q_out[ATJUP_S_COUNT + 2];
    void* acc[ATJUP_S_COUNT + 2];
    // FP64: the time-level-n copies and the live fields (the non-integrated copy)
    const double* q_n[ATJUP_S_COUNT + 2];
    const double* q_live[ATJUP_S_COUNT + 2];
    // frozen inputs
    const double* sprec[9];
    const double *mf_h2s, *mf_nh3, *mf_nh4sh, *fluxlim;
    const double *nue, *rho_mix;
    const double* vel_star;            // [jm][KP]
    const float* layer_h;              // [im]
    const int32_t* topo;               // [jm * km]
    // closure outputs
    double *prod, *tke_source, *dis_source;
    const uint8_t* flags;
    const GeoIJ* geo;
    int im, jm, km, KP, stage;
    // FP64 step: the species keep no accumulator. Stage s's right-hand side is recovered from the
    // next stage input as (X_{s+1} - y_n) / c_s (exact: X_{s+1} lies within a factor 2 of y_n,
    // so the subtraction is exact, Sterbenz), so stage 3 reads X1 and X2 beside its own input X3
    // instead of one accumulator that stages 0-2 would each write and stages 1-2 read.
    int acc_free;
    const double* x1[ATJUP_S_COUNT];   // X1, X2 of the species (stage 3, acc_free)
    const double* x2[ATJUP_S_COUNT];
    double inv_c_half, inv_dt;         // 1 / c of stages 0 and 1 (2 / dt) and of stage 2 (1 / dt)
    double c_in, wgt, dt, one_sixth;
    double inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
    double coef[ATJUP_S_COUNT];        // species_diff_scale / (sc re)
    double precip_coupling, chemical_reaction, turb_coupling;
    double stokes_pre, rg_nh4sh, mue_mix;  // (2/9) r_p r_p, computed in the reference's order
    double inv_re, L_m, u_0, t_ref, g, cp_mix, nue_max, tke_max_nd, re_turb, turb_buoy_prt;
    int has_nue, turb_model, turb_buoy;
};

template <typename R> __device__ __forceinline__ R dmax(R a, R b) { return a < b ? b : a; }   // std::max
template <typename R> __device__ __forceinline__ R dmin(R a, R b) { return b < a ? b : a; }   // std::min

__device__ __forceinline__ double safe_clamp(double v, double lo, double hi) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    if ((b & 0x7FF0000000000000ULL) == 0x7FF0000000000000ULL) return lo;
    return (v < lo) ? lo : ((v > hi) ? hi : v);
}

// float m_layer_heights [km]: get_layer_height (-1 out of range), layer_thickness_m
__device__ __forceinline__ double layer_h(const PhysStage& a, int i) {
    if (i < 0 || i > a.im - 1) return (double)(-1.0f);
    return (double)a.layer_h[i];
}
__device__ __forceinline__ double layer_dz_m(const PhysStage& a, int i) {
    if (i < 0 || i > a.im - 2) return -1.0;
    return (double)(a.layer_h[i + 1] - a.layer_h[i]) * 1.0e3;
}

struct Cell {
    size_t c, cip, cim, cjp, cjm, ckp, ckm;
};

// The cell and its six neighbours; the i and j neighbours of the block's faces are clamped to the
// cell itself (those cells are never integrated: their loads only have to stay in bounds).
__device__ __forceinline__ Cell cell_of(const PhysStage& a, int i, int j, int k) {
    Cell x;
    const size_t row = ((size_t)i * a.jm + j) * a.KP, plane = (size_t)a.jm * a.KP;
    const int ke = (k >= a.km - 2) ? 0 : k + 1, kw = (k == 0) ? a.km - 2 : k - 1;
    x.c = row + k;
    x.cip = (i < a.im - 1) ? x.c + plane : x.c;
    x.cim = (i > 0) ? x.c - plane : x.c;
    x.cjp = (j < a.jm - 1) ? x.c + a.KP : x.c;
    x.cjm = (j > 0) ? x.c - a.KP : x.c;
    x.ckp = row + ke;
    x.ckm = row + kw;
    return x;
}

// RK bookkeeping of one scalar at an integrated cell (RungeKutta_Jup_Turb.cpp:425-490, 493-568).
// The accumulator is summed in R and stored as TA; the next stage input and the final update are
// formed in FP64 from the FP64 time-level-n value, then clamped, then stored as TO.
template <typename TO, typename TA, typename R>
__device__ __forceinline__ void rk_update(const PhysStage& a, int s, size_t c, R rhs, R acc_in,
                                          double qn) {
    const R acc = (a.stage == 0) ? (R)a.wgt * rhs : acc_in + (R)a.wgt * rhs;
    if (a.stage < 3) {
        static_cast<TA*>(a.acc[s])[c] = (TA)acc;
        double x = qn + (double)((R)a.c_in * rhs);
        if (s == ATJUP_S_COUNT) x = safe_clamp(x, 0.0, a.tke_max_nd);          // k*
        else if (s == ATJUP_S_COUNT + 1) x = dmax(1.0e-10, x);                 // omega*
        static_cast<TO*>(a.q_out[s])[c] = (TO)x;
    } else {
        double x = qn + a.dt * (double)acc * a.one_sixth;
        if (s == ATJUP_S_COUNT) x = safe_clamp(x, 0.0, a.tke_max_nd);
        else if (s == ATJUP_S_COUNT + 1) x = dmax(1.0e-10, x);
        else if (s == ATJUP_S_NH4SH) x = (x < 0.0) ? 0.0 : x;                  // keeps NaN, -0
        else x = dmax(0.0, x);
        static_cast<TO*>(a.q_out[s])[c] = (TO)x;
    }
}

__device__ __forceinline__ int precip_slot(int s) {
    switch (s) {
    case ATJUP_S_H2O: return 0;
    case ATJUP_S_H2O_CLOUD: return 1;
    case ATJUP_S_H2O_ICE: return 2;
    case ATJUP_S_NH3: return 3;
    case ATJUP_S_NH3_CLOUD: return 4;
    case ATJUP_S_NH3_ICE: return 5;
    case ATJUP_S_CH4: return 6;
    case ATJUP_S_CH4_CLOUD: return 7;
    case ATJUP_S_CH4_ICE: return 8;
    default: return -1;
    }
}

// Template arguments of the stage kernels: TI the stage input's storage (velocities, temperature,
// scalars), TO the next stage input's (stage 3: the live FP64 field), TA the accumulators', R the
// arithmetic of the right-hand side. The FP64 step is <double, double, double, double>; the mixed
// step keeps FP32 stage buffers and accumulators and FP32 arithmetic: stage 0 <double, float,
// float, float> (it reads the live fields), stages 1-2 <float, float, float, float>, stage 3
// <float, double, float, float>.

// One thread per cell, the eleven species in turn (an unrolled loop: each species' index, sources
// and coefficients are compile-time): what the species share -- the cell's indices, its flags,
// u, v, w, nue and the eddy diffusivity nue_t / 0.9, the row's geometry -- is read and formed once
// per cell. Each species reads its own 7-point stencil (coalesced along k), its FP64
// time-level-n value, its accumulator (or, FP64 stage 3, X1 and X2) and its frozen sources.
// blockIdx.y * blockDim.y + threadIdx.y = j, blockIdx.x * blockDim.x + threadIdx.x = k,
// blockIdx.z = i.
template <typename R>
struct CellShared {
    R u0, v_invrm, w_invrs, two_inv_rm, inv_rm2, ci, is2, nue_t_s;
    double rho;
};

// The right-hand side of species S at a cell from its stencil and sources
// (RHS_Jup_Turb.cpp species part), in R.
template <int S, typename R>
__device__ __forceinline__ R species_rhs(const PhysStage& a, const CellShared<R>& z, R f0, R fip,
                                         R fim, R fjp, R fjm, R fkp, R fkm, double src0,
                                         double src1) {
    const R d1r = (fip - fim) * (R)a.inv_2dr;
    const R d2r = (fip - (R)2 * f0 + fim) * (R)a.inv_dr2;
    const R d1t = (fjp - fjm) * (R)a.inv_2dthe;
    const R d2t = (fjp - (R)2 * f0 + fjm) * (R)a.inv_dthe2;
    const R d1p = (fkp - fkm) * (R)a.inv_2dphi;
    const R d2p = (fkp - (R)2 * f0 + fkm) * (R)a.inv_dphi2;
    const R transport = z.u0 * d1r + z.v_invrm * d1t + z.w_invrs * d1p;
    const R diffusion = d2r + d1r * z.two_inv_rm + d2t * z.inv_rm2 + d1t * z.ci + d2p * z.is2;
    const R coef = (R)a.coef[S] + z.nue_t_s;
    R r;
    if constexpr (S == ATJUP_S_H2S) {
        r = -transport + diffusion * coef + (R)(a.chemical_reaction * src0);
    } else if constexpr (S == ATJUP_S_NH3) {
        r = -transport + diffusion * coef + (R)(a.chemical_reaction * src0) +
            (R)(a.precip_coupling * src1);
    } else if constexpr (S == ATJUP_S_NH4SH) {
        const double v_stokes = a.stokes_pre * (a.rg_nh4sh - z.rho) * a.g / a.mue_mix;
        r = -transport + (R)src0 + diffusion * coef + (R)(a.chemical_reaction * src1) +
            (R)(v_stokes / a.u_0) * d1r;
    } else {
        r = -transport + diffusion * coef + (R)(a.precip_coupling * src0);
    }
    return r;
}

// FP64 step, no accumulator: the next stage input, or at stage 3 the clamped result from the
// right-hand sides recovered from X1, X2, X3 (f0)
template <int S>
__device__ __forceinline__ double species_acc_free_out(const PhysStage& a, double r, double f0,
                                                       double qn, double x1, double x2) {
    if (a.stage < 3) return qn + a.c_in * r;
    const double k1 = (x1 - qn) * a.inv_c_half, k2 = (x2 - qn) * a.inv_c_half;
    const double k3 = (f0 - qn) * a.inv_dt;
    const double acc = ((k1 + 2.0 * k2) + 2.0 * k3) + r;
    const double q = qn + a.dt * acc * a.one_sixth;
    return (S == ATJUP_S_NH4SH) ? ((q < 0.0) ? 0.0 : q) : dmax(0.0, q);
}

template <int S>
__device__ __forceinline__ const double* species_src0(const PhysStage& a) {
    if constexpr (S == ATJUP_S_H2S) return a.mf_h2s;
    else if constexpr (S == ATJUP_S_NH3) return a.mf_nh3;
    else if constexpr (S == ATJUP_S_NH4SH) return a.fluxlim;
    else return a.sprec[precip_slot(S)];
}
template <int S>
__device__ __forceinline__ const double* species_src1(const PhysStage& a) {
    if constexpr (S == ATJUP_S_NH3) return a.sprec[3];
    else if constexpr (S == ATJUP_S_NH4SH) return a.mf_nh4sh;
    else return nullptr;
}

// One species' inputs at the cell. The next species' are loaded before this one's results are
// stored: the stores may alias the loads as far as the compiler knows, so only this order lets
// two species' loads be in flight at once.
template <typename R>
struct SpIn {
    R f0, fip, fim, fjp, fjm, fkp, fkm, acc_in;
    double qn, x1, x2, src0, src1;
};

template <int S, typename TI, typename TA, typename R>
__device__ __forceinline__ SpIn<R> species_load(const PhysStage& a, const Cell& x) {
    SpIn<R> v;
    const size_t c = x.c;
    const TI* F = static_cast<const TI*>(a.q_in[S]);
    v.f0 = (R)F[c]; v.fip = (R)F[x.cip]; v.fim = (R)F[x.cim]; v.fjp = (R)F[x.cjp];
    v.fjm = (R)F[x.cjm]; v.fkp = (R)F[x.ckp]; v.fkm = (R)F[x.ckm];
    v.qn = a.q_n[S][c];
    v.acc_in = (R)0;
    v.x1 = 0.0;
    v.x2 = 0.0;
    if (a.acc_free) {
        if (a.stage == 3) { v.x1 = a.x1[S][c]; v.x2 = a.x2[S][c]; }
    } else if (a.stage > 0) {
        v.acc_in = (R)static_cast<const TA*>(a.acc[S])[c];
    }
    const double* s1 = species_src1<S>(a);
    v.src0 = species_src0<S>(a)[c];
    v.src1 = s1 ? s1[c] : 0.0;
    return v;
}

template <int S, typename TO, typename TA, typename R>
__device__ __forceinline__ void species_finish(const PhysStage& a, size_t c, const CellShared<R>& z,
                                               const SpIn<R>& v) {
    const R r = species_rhs<S, R>(a, z, v.f0, v.fip, v.fim, v.fjp, v.fjm, v.fkp, v.fkm, v.src0, v.src1);
    if (a.acc_free) {
        static_cast<TO*>(a.q_out[S])[c] =
            (TO)species_acc_free_out<S>(a, (double)r, (double)v.f0, v.qn, v.x1, v.x2);
        return;
    }
    rk_update<TO, TA, R>(a, S, c, r, v.acc_in, v.qn);
}

template <int S, typename TI, typename TO, typename TA, typename R>
__device__ __forceinline__ void species_all(const PhysStage& a, const Cell& x,
                                            const CellShared<R>& z, const SpIn<R>& cur) {
    if constexpr (S + 1 < ATJUP_S_COUNT) {
        const SpIn<R> nxt = species_load<S + 1, TI, TA, R>(a, x);
        species_finish<S, TO, TA, R>(a, x.c, z, cur);
        species_all<S + 1, TI, TO, TA, R>(a, x, z, nxt);
    } else {
        species_finish<S, TO, TA, R>(a, x.c, z, cur);
    }
}

// Three blocks per SM (at most 80 registers): with two species' loads in flight the FP64 form
// needs 96 registers unbounded (two blocks per SM) and spills heavily at 64 (four blocks); the
// step measured 6.77 ms at 80 against 7.06 at 96, 7.14 at 64 and 6.89 without the early loads.
template <typename TI, typename TO, typename TA, typename R>
__global__ void __launch_bounds__(256, 3) species_stage_kernel(PhysStage a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= a.km || j >= a.jm) return;
    const Cell x = cell_of(a, i, j, k);
    const size_t c = x.c;
    // the loads the species share, issued with the flag before the integrated-cell test
    const uint8_t fl = a.flags[c];
    const R u0 = (R)static_cast<const TI*>(a.u)[c];
    const R v0 = (R)static_cast<const TI*>(a.v)[c];
    const R w0 = (R)static_cast<const TI*>(a.w)[c];
    const double nv = a.has_nue ? a.nue[c] : 0.0;
    const double rho = a.rho_mix[c];
    if (!(fl & NB_INT)) {
        // the cell keeps its live values through the step
        if (a.stage < 3) {
#pragma unroll
            for (int s = 0; s < ATJUP_S_COUNT; s++)
                static_cast<TO*>(a.q_out[s])[c] = (TO)a.q_live[s][c];
        }
        return;
    }
    const GeoIJ& g = a.geo[(size_t)i * a.jm + j];
    CellShared<R> z;
    z.u0 = u0;
    z.v_invrm = v0 * (R)g.inv_rm;
    z.w_invrs = w0 * (R)g.inv_rmsinthe;
    z.two_inv_rm = (R)2 * (R)g.inv_rm;
    z.inv_rm2 = (R)g.inv_rm2;
    z.ci = (R)g.costhe_inv_rm2sinthe;
    z.is2 = (R)g.inv_rm2sinthe2;
    double nue_t64 = 0.0;
    if (a.has_nue && a.turb_coupling != 0.0 && isfinite(nv)) nue_t64 = a.turb_coupling * dmax(0.0, nv);
    const R nue_t = (R)nue_t64;
    z.nue_t_s = nue_t / (R)0.9;
    z.rho = rho;
    species_all<0, TI, TO, TA, R>(a, x, z, species_load<0, TI, TA, R>(a, x));
}

// k*, omega*: transport, diffusion with the model's coefficients, and the closure sources
// (RHS_Jup_Turb.cpp:257-303, 736-998, 1399-1452). One instantiation per closure model, so that
// each holds the registers of its own branch only. Three blocks per SM (at most 80 registers: the
// k-omega SST form spilled 172 bytes at 64; the step measured 6.70 ms against 6.72 at 64 and 6.82
// at 128).
template <int MODEL, typename TI, typename TO, typename TA, typename R>
__global__ void __launch_bounds__(256, 3) closure_stage_kernel(PhysStage a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= a.km || j >= a.jm) return;
    const int ST = ATJUP_S_COUNT, SD = ATJUP_S_COUNT + 1;
    // Every load is issued before the integrated-cell test (one memory round trip): the
    // neighbour addresses are clamped into the block, so boundary cells read only their own
    // cell before the test sends them to the copy below.
    const Cell x = cell_of(a, i, j, k);
    const uint8_t fl = a.flags[x.c];
    const TI* TK = static_cast<const TI*>(a.q_in[ST]);
    const TI* DS = static_cast<const TI*>(a.q_in[SD]);
    const TI* Us = static_cast<const TI*>(a.u);
    const TI* Vs = static_cast<const TI*>(a.v);
    const TI* Ws = static_cast<const TI*>(a.w);
    const R tk0 = (R)TK[x.c], ds0 = (R)DS[x.c];
    const R tip_ = (R)TK[x.cip], tim_ = (R)TK[x.cim], tjp_ = (R)TK[x.cjp], tjm_ = (R)TK[x.cjm];
    const R tkp_ = (R)TK[x.ckp], tkm_ = (R)TK[x.ckm];
    const R dip_ = (R)DS[x.cip], dim_ = (R)DS[x.cim], djp_ = (R)DS[x.cjp], djm_ = (R)DS[x.cjm];
    const R dkp_ = (R)DS[x.ckp], dkm_ = (R)DS[x.ckm];
    const R u0 = (R)Us[x.c], v0 = (R)Vs[x.c], w0 = (R)Ws[x.c];
    const R uip = (R)Us[x.cip], uim = (R)Us[x.cim], vip = (R)Vs[x.cip], vim = (R)Vs[x.cim];
    const R wip = (R)Ws[x.cip], wim = (R)Ws[x.cim];
    const R ujp = (R)Us[x.cjp], ujm = (R)Us[x.cjm], vjp = (R)Vs[x.cjp], vjm = (R)Vs[x.cjm];
    const R wjp = (R)Ws[x.cjp], wjm = (R)Ws[x.cjm];
    const R ukp = (R)Us[x.ckp], ukm = (R)Us[x.ckm], vkp = (R)Vs[x.ckp], vkm = (R)Vs[x.ckm];
    const R wkp = (R)Ws[x.ckp], wkm = (R)Ws[x.ckm];
    const double nv = a.nue[x.c];
    const int32_t topo = a.topo[(size_t)j * a.km + k];
    if (!(fl & NB_INT)) {
        if (a.stage < 3) {
            static_cast<TO*>(a.q_out[ST])[x.c] = (TO)a.q_live[ST][x.c];
            static_cast<TO*>(a.q_out[SD])[x.c] = (TO)a.q_live[SD][x.c];
        }
        return;
    }
    const GeoIJ& g = a.geo[(size_t)i * a.jm + j];
    const R inv_rm = (R)g.inv_rm, inv_rmsinthe = (R)g.inv_rmsinthe;
    // the solid-face mirror (RHS_Jup_Turb.cpp:257-303): a solid neighbour reads as the cell
    const R tip = (fl & NB_IP) ? tk0 : tip_, tim = (fl & NB_IM) ? tk0 : tim_;
    const R tjp = (fl & NB_JP) ? tk0 : tjp_, tjm = (fl & NB_JM) ? tk0 : tjm_;
    const R tkp = (fl & NB_KP) ? tk0 : tkp_, tkm = (fl & NB_KM) ? tk0 : tkm_;
    const R dip = (fl & NB_IP) ? ds0 : dip_, dim = (fl & NB_IM) ? ds0 : dim_;
    const R djp = (fl & NB_JP) ? ds0 : djp_, djm = (fl & NB_JM) ? ds0 : djm_;
    const R dkp = (fl & NB_KP) ? ds0 : dkp_, dkm = (fl & NB_KM) ? ds0 : dkm_;
    const R i2r = (R)a.inv_2dr, i2t = (R)a.inv_2dthe, i2p = (R)a.inv_2dphi;
    const R dtkedr = (tip - tim) * i2r, d2tkedr2 = (tip - (R)2 * tk0 + tim) * (R)a.inv_dr2;
    const R ddisdr = (dip - dim) * i2r, d2disdr2 = (dip - (R)2 * ds0 + dim) * (R)a.inv_dr2;
    const R dtkedthe = (tjp - tjm) * i2t;
    const R d2tkedthe2 = (tjp - (R)2 * tk0 + tjm) * (R)a.inv_dthe2;
    const R ddisdthe = (djp - djm) * i2t;
    const R d2disdthe2 = (djp - (R)2 * ds0 + djm) * (R)a.inv_dthe2;
    const R dtkedphi = (tkp - tkm) * i2p;
    const R d2tkedphi2 = (tkp - (R)2 * tk0 + tkm) * (R)a.inv_dphi2;
    const R ddisdphi = (dkp - dkm) * i2p;
    const R d2disdphi2 = (dkp - (R)2 * ds0 + dkm) * (R)a.inv_dphi2;

    const R dudr = (uip - uim) * i2r;
    const R dvdr = (vip - vim) * i2r;
    const R dwdr = (wip - wim) * i2r;
    const R dudthe = (ujp - ujm) * i2t;
    const R dvdthe = (vjp - vjm) * i2t;
    const R dwdthe = (wjp - wjm) * i2t;
    const R dudphi = (ukp - ukm) * i2p;
    const R dvdphi = (vkp - vkm) * i2p;
    const R dwdphi = (wkp - wkm) * i2p;
    const R v_invrm = v0 * inv_rm;
    const R w_invrs = w0 * inv_rmsinthe;
    const R two_inv_rm = (R)2 * inv_rm;
    const R transport_tke = u0 * dtkedr + v_invrm * dtkedthe + w_invrs * dtkedphi;
    const R transport_dis = u0 * ddisdr + v_invrm * ddisdthe + w_invrs * ddisdphi;
    const R diffusion_tke = d2tkedr2 + dtkedr * two_inv_rm + d2tkedthe2 * (R)g.inv_rm2 +
                            dtkedthe * (R)g.costhe_inv_rm2sinthe + d2tkedphi2 * (R)g.inv_rm2sinthe2;
    const R diffusion_dis = d2disdr2 + ddisdr * two_inv_rm + d2disdthe2 * (R)g.inv_rm2 +
                            ddisdthe * (R)g.costhe_inv_rm2sinthe + d2disdphi2 * (R)g.inv_rm2sinthe2;

    const R C_nue = (R)0.028, dis_min = (R)1.0e-10;
    const double nue_gas_phys = 1.8e-5;
    const double L_m = a.L_m;
    const R nue_here = isfinite(nv) ? (R)dmax(0.0, nv) : (R)0;
    const R tke_s = dmax(tk0, dis_min);
    const R dis_s = dmax(ds0, dis_min);
    const R dudr_s = dudr, dvdr_s = dvdr, dwdr_s = dwdr;
    const R dudthe_s = dudthe * inv_rm, dvdthe_s = dvdthe * inv_rm;
    const R dwdthe_s = dwdthe * inv_rm;
    const R dudphi_s = dudphi * inv_rmsinthe, dvdphi_s = dvdphi * inv_rmsinthe;
    const R dwdphi_s = dwdphi * inv_rmsinthe;
    const R dtkedthe_s = dtkedthe * inv_rm, ddisdthe_s = ddisdthe * inv_rm;
    const R dtkedphi_s = dtkedphi * inv_rmsinthe, ddisdphi_s = ddisdphi * inv_rmsinthe;
    const R grad_dot = dtkedr * ddisdr + dtkedthe_s * ddisdthe_s + dtkedphi_s * ddisdphi_s;
    R cnue = (MODEL == ATJUP_TURB_K_EPSILON) ? C_nue * tke_s * tke_s / dis_s : tke_s / dis_s;
    cnue = dmin(cnue, (R)a.nue_max);
    const R c23 = (R)0.66667, two = (R)2;
    const R der = c23 * (dudr_s + dvdthe_s + dwdphi_s);
    const R P_full = dmax((R)0,
          (cnue * (two * dudr_s - der) - c23 * tk0) * dudr_s
        + (cnue * (dudthe_s + dvdr_s)) * dudthe_s
        + (cnue * (dudphi_s + dwdr_s)) * dudphi_s
        + (cnue * (two * dvdthe_s - der) - c23 * tk0) * dvdthe_s
        + (cnue * (dvdr_s + dudthe_s)) * dvdr_s
        + (cnue * (dvdphi_s + dwdthe_s)) * dvdphi_s
        + (cnue * (two * dwdphi_s - der) - c23 * tk0) * dwdphi_s
        + (cnue * (dwdr_s + dudphi_s)) * dwdr_s
        + (cnue * (dwdthe_s + dvdphi_s)) * dwdthe_s);

    const double y_mount = layer_h(a, topo) * 1.0e3;
    const double dz_layer = dmax(1.0, layer_dz_m(a, i - 1 > 0 ? i - 1 : 0));
    const double y_phys = dmax(layer_h(a, i) * 1.0e3 - y_mount, dz_layer);
    const R y_star = (R)(y_phys / L_m);
    const R inv_re = (R)a.inv_re;

    R dtre, ddre, tke_src, dis_src, c_w_prod;
    if (MODEL == ATJUP_TURB_K_EPSILON) {                      // Chien 1982
        const R sig_k = (R)1.0, sig_w = (R)1.3, C_eps_1 = (R)1.35, C_eps_2 = (R)1.80;
        dtre = inv_re + nue_here / sig_k;
        ddre = inv_re + nue_here / sig_w;
        // the wall-damping exponentials in FP64: their arguments overflow FP32 near dis_min
        const double d_plus = y_phys * a.vel_star[(size_t)j * a.KP + k] / nue_gas_phys;
        const double tke_d = (double)tke_s, dis_d = (double)dis_s;
        const double Re_T = tke_d * tke_d * a.u_0 * L_m / (dis_d * nue_gas_phys);
        const R f_2 = (R)(1.0 - 0.4 / 1.8 * exp(-Re_T * Re_T / 36.0));
        const R y_star2 = y_star * y_star;
        const R L_k = -(R)2 * tk0 / y_star2;
        const R L_w = (R)(-2.0 * (double)ds0 / (double)y_star2 * exp(-0.5 * d_plus));
        const R P_w = C_eps_1 * ds0 / tke_s * P_full;
        const R Y_w = C_eps_2 * f_2 * ds0 * ds0 / tke_s;
        tke_src = P_full - ds0 + L_k / (R)a.re_turb;
        dis_src = P_w - Y_w + L_w / (R)a.re_turb;
        c_w_prod = C_eps_1;
    } else if (MODEL == ATJUP_TURB_K_OMEGA) {                 // Wilcox
        const R sig_k = (R)0.6, sig_w = (R)0.5, bet_star = (R)0.09, gam = (R)0.52;
        const double bet_0 = 0.0708;
        dtre = inv_re + sig_k * nue_here;
        ddre = inv_re + sig_w * nue_here;
        const R S11 = dudr_s, S22 = dvdthe_s, S33 = dwdphi_s;
        const R S12 = (R)0.5 * (dudthe_s + dvdr_s);
        const R S13 = (R)0.5 * (dudphi_s + dwdr_s);
        const R S23 = (R)0.5 * (dvdphi_s + dwdthe_s);
        const R S_mag = sqrt((R)2 * (S11 * S11 + S22 * S22 + S33 * S33 +
                                     (R)2 * (S12 * S12 + S13 * S13 + S23 * S23)));
        const R W12 = dudthe_s - dvdr_s;
        const R W13 = dudphi_s - dwdr_s;
        const R W23 = dvdphi_s - dwdthe_s;
        const R Omega = sqrt(W12 * W12 + W13 * W13 + W23 * W23);
        // the vortex-stretching ratio in FP64: (0.09 omega*)^3 underflows FP32 near dis_min
        const double bd = 0.09 * (double)dis_s;
        const double chi_w = fabs((double)Omega * (double)Omega * (double)S_mag / (bd * bd * bd));
        const double f_bet = (1.0 + 85.0 * chi_w) / (1.0 + 100.0 * chi_w);
        const R bet_wc = (R)(bet_0 * f_bet);
        const R sig_d = (grad_dot <= (R)0) ? (R)0 : (R)0.125;
        const R P_k = dmin(P_full, (R)20 * bet_star * tke_s * dis_s);
        const R Y_k = bet_star * tke_s * dis_s;
        const R P_w = gam * dis_s / tke_s * P_k;
        const R Y_w = bet_wc * dis_s * dis_s;
        const R D_w = sig_d / dis_s * grad_dot;
        tke_src = P_k - Y_k;
        dis_src = P_w - Y_w + D_w;
        c_w_prod = gam;
    } else {                                                   // SST, Menter 1994
        const R bet_star = (R)0.09, sig_k1 = (R)1.176, sig_k2 = (R)1.0, sig_w1 = (R)2.0;
        const R sig_w2 = (R)1.168;
        const R bet1 = (R)0.0333, bet2 = (R)0.0368, gam1 = (R)0.413, gam2 = (R)0.2;
        const R nue_air_nd = (R)(nue_gas_phys / (a.u_0 * L_m));
        const R CD_kw = dmax((R)2 * sig_w2 / dis_s * grad_dot, (R)1.0e-20);
        const R arg1 = dmin(dmax(sqrt(dmax(tk0, (R)0)) / (bet_star * dis_s * y_star),
                                 (R)500 * nue_air_nd / (y_star * y_star * dis_s)),
                            (R)4 * sig_w2 * tke_s / (CD_kw * y_star * y_star));
        const R a2 = arg1 * arg1;
        const R F1 = tanh(a2 * a2);                                          // pow(arg1, 4)
        const R one = (R)1;
        const R sig_k = F1 * sig_k1 + (one - F1) * sig_k2;
        const R sig_w = F1 * sig_w1 + (one - F1) * sig_w2;
        dtre = inv_re + nue_here / sig_k;
        ddre = inv_re + nue_here / sig_w;
        const R P_k = dmin(P_full, (R)20 * bet_star * tke_s * dis_s);
        const R Y_k = bet_star * tke_s * dis_s;
        const R P_w = (F1 * gam1 + (one - F1) * gam2) * P_k * dis_s / tke_s;
        const R Y_w = (F1 * bet1 + (one - F1) * bet2) * dis_s * dis_s;
        const R D_w = (R)2 * (one - F1) * sig_w2 / dis_s * grad_dot;
        tke_src = P_k - Y_k;
        dis_src = P_w - Y_w + D_w;
        c_w_prod = F1 * gam1 + (one - F1) * gam2;
    }
    if (a.turb_buoy) {                                         // RHS_Jup_Turb.cpp:963-981
        const TI* Ts = static_cast<const TI*>(a.t);
        const int ip = (i + 1 < a.im - 1) ? i + 1 : a.im - 1, imn = (i - 1 > 0) ? i - 1 : 0;
        const double dz_m = (layer_h(a, ip) - layer_h(a, imn)) * 1.0e3;
        const size_t rs = (size_t)a.jm * a.KP;
        const double T_K = dmax((double)Ts[x.c] * a.t_ref, 1.0);
        const double dTdz = ((double)Ts[x.c + (ip - i) * rs] - (double)Ts[x.c - (i - imn) * rs]) *
                            a.t_ref / dmax(dz_m, 1.0);
        const double N2 = a.g / T_K * (dTdz + a.g / a.cp_mix);
        const double tscale = L_m / a.u_0;
        const double G_b = -((double)cnue / a.turb_buoy_prt) * N2 * tscale * tscale;
        if (isfinite(G_b)) {
            tke_src += (R)G_b;
            dis_src += c_w_prod * dis_s / tke_s * (R)dmax(G_b, 0.0);
        }
    }
    const R tke_src_max = (R)20 * tke_s * dis_s;
    const R dis_src_max = (R)20 * dis_s * dis_s;
    if (!isfinite(tke_src)) tke_src = (R)0;
    if (!isfinite(dis_src)) dis_src = (R)0;
    tke_src = dmax(-tke_src_max, dmin(tke_src_max, tke_src));
    dis_src = dmax(-dis_src_max, dmin(dis_src_max, dis_src));
    if (a.stage == 3) {
        a.prod[x.c] = (double)P_full;
        a.tke_source[x.c] = (double)tke_src;
        a.dis_source[x.c] = (double)dis_src;
    }
    // the accumulators and n copies are read here, not with the stencil: read early they hold
    // four more registers (8 in FP64) through the whole source computation
    const R acc_t = (a.stage == 0) ? (R)0 : (R)static_cast<const TA*>(a.acc[ST])[x.c];
    const R acc_d = (a.stage == 0) ? (R)0 : (R)static_cast<const TA*>(a.acc[SD])[x.c];
    rk_update<TO, TA, R>(a, ST, x.c, -transport_tke + diffusion_tke * dtre + tke_src, acc_t,
                         a.q_n[ST][x.c]);
    rk_update<TO, TA, R>(a, SD, x.c, -transport_dis + diffusion_dis * ddre + dis_src, acc_d,
                         a.q_n[SD][x.c]);
}

}  // namespace

// Field ids of the transported scalars in ATJUP_S_* order, then k*, omega*.
const int kScalarField[ATJUP_S_COUNT + 2] = {
    ATJUP_F_H2O, ATJUP_F_H2O_CLOUD, ATJUP_F_H2O_ICE, ATJUP_F_H2S, ATJUP_F_NH3,
    ATJUP_F_NH3_CLOUD, ATJUP_F_NH3_ICE, ATJUP_F_CH4, ATJUP_F_CH4_CLOUD, ATJUP_F_CH4_ICE,
    ATJUP_F_NH4SH, ATJUP_F_TKE, ATJUP_F_DIS};

namespace {
PhysStage stage_args(AtjupCtx* c, int stage, const void* const* vin) {
    const AtjupParams& P = c->P;
    const AtjupPhysics& H = c->phys;
    PhysStage a{};
    a.u = vin[1];
    a.v = vin[2];
    a.w = vin[3];
    for (int s = 0; s < ATJUP_S_COUNT + 2; s++) {
        const int id = kScalarField[s];
        double* live = c->f[id];
        // the stage buffers hold doubles, or floats in their first half in the mixed step; the
        // FP64 species keep X1, X2 to the end and put X3 where the accumulator would be
        const bool af = (s < ATJUP_S_COUNT) && c->step_prec != ATJUP_PREC_MIXED;
        const void* in[4] = {live, c->S1[s], c->S2[s], af ? (const void*)c->Sacc[s] : c->S1[s]};
        void* out[4] = {c->S1[s], c->S2[s], af ? (void*)c->Sacc[s] : c->S1[s], live};
        a.q_in[s] = in[stage];
        a.q_out[s] = out[stage];
        if (s < ATJUP_S_COUNT) {
            a.x1[s] = c->S1[s];
            a.x2[s] = c->S2[s];
        }
        a.q_n[s] = c->fn[id];
        a.acc[s] = c->Sacc[s];
        a.q_live[s] = live;
    }
    const int sp[9] = {ATJUP_F_S_PRECIP_H2O, ATJUP_F_S_PRECIP_H2O_CLOUD, ATJUP_F_S_PRECIP_H2O_ICE,
                       ATJUP_F_S_PRECIP_NH3, ATJUP_F_S_PRECIP_NH3_CLOUD, ATJUP_F_S_PRECIP_NH3_ICE,
                       ATJUP_F_S_PRECIP_CH4, ATJUP_F_S_PRECIP_CH4_CLOUD, ATJUP_F_S_PRECIP_CH4_ICE};
    for (int q = 0; q < 9; q++) a.sprec[q] = c->f[sp[q]];
    a.mf_h2s = c->f[ATJUP_F_MASSFLUX_H2S];
    a.mf_nh3 = c->f[ATJUP_F_MASSFLUX_NH3];
    a.mf_nh4sh = c->f[ATJUP_F_MASSFLUX_NH4SH];
    a.fluxlim = c->f[ATJUP_F_FLUXLIM_NH4SH];
    a.nue = c->f[ATJUP_F_NUE];
    a.rho_mix = c->f[ATJUP_F_RHO_MIX];
    a.t = vin[0];                       // the stage input temperature (buoyancy production)
    a.vel_star = c->f2[ATJUP_F2_VEL_STAR];
    a.layer_h = c->layer_h;
    a.topo = c->topo;
    a.prod = c->f[ATJUP_F_PROD];
    a.tke_source = c->f[ATJUP_F_TKE_SOURCE];
    a.dis_source = c->f[ATJUP_F_DIS_SOURCE];
    a.flags = c->nbflags;
    a.geo = c->geo;
    a.im = P.im; a.jm = P.jm; a.km = P.km; a.KP = c->KP; a.stage = stage;
    a.acc_free = (c->step_prec != ATJUP_PREC_MIXED) ? 1 : 0;
    a.inv_c_half = 2.0 / P.dt;
    a.inv_dt = 1.0 / P.dt;
    a.c_in = (stage == 0 || stage == 1) ? 0.5 * P.dt : (stage == 2 ? P.dt : 0.0);
    a.wgt = (stage == 0 || stage == 3) ? 1.0 : 2.0;
    a.dt = P.dt;
    a.one_sixth = 1.0 / 6.0;
    a.inv_2dr = 1.0 / (2.0 * P.dr);
    a.inv_2dthe = 1.0 / (2.0 * P.dthe);
    a.inv_2dphi = 1.0 / (2.0 * P.dphi);
    a.inv_dr2 = 1.0 / (P.dr * P.dr);
    a.inv_dthe2 = 1.0 / (P.dthe * P.dthe);
    a.inv_dphi2 = 1.0 / (P.dphi * P.dphi);
    const double sc[ATJUP_S_COUNT] = {H.sc_h2o, H.sc_h2o, H.sc_h2o, H.sc_h2s, H.sc_nh3, H.sc_nh3,
                                      H.sc_nh3, H.sc_ch4, H.sc_ch4, H.sc_ch4, H.sc_nh4sh};
    for (int s = 0; s < ATJUP_S_COUNT; s++) a.coef[s] = H.species_diff_scale / (sc[s] * P.re);
    a.precip_coupling = P.precip_coupling;
    a.chemical_reaction = H.chemical_reaction;
    a.turb_coupling = P.turb_coupling;
    a.stokes_pre = (2.0 / 9.0) * H.r_p_nh4sh * H.r_p_nh4sh;
    a.rg_nh4sh = H.rg_nh4sh;
    a.mue_mix = H.mue_mix;
    a.inv_re = 1.0 / P.re;
    a.L_m = P.L_atm * 1.0e3;
    a.u_0 = P.u_0;
    a.t_ref = P.t_ref;
    a.g = P.g;
    a.cp_mix = P.cp_mix;
    a.nue_max = H.nue_max_phys / (P.u_0 * a.L_m);
    a.tke_max_nd = H.tke_max_phys / (P.u_0 * P.u_0);
    a.re_turb = H.re_turb;
    a.turb_buoy_prt = H.turb_buoy_prt;
    a.has_nue = P.has_nue;
    a.turb_model = H.turb_model;
    a.turb_buoy = H.turb_buoy;
    return a;
}
}  // namespace

template <typename TI, typename TO, typename TA, typename R>
static int launch_typed(AtjupCtx* c, const PhysStage& a, int what, cudaStream_t st) {
    const AtjupParams& P = c->P;
    const dim3 block(128, 2);
    const dim3 grid((P.km + 127) / 128, (P.jm + 1) / 2, P.im);
    if (what == 0) {
        species_stage_kernel<TI, TO, TA, R><<<grid, block, 0, st>>>(a);
        c->launches++;
        ATJUP_CHECK_LAUNCH("species_stage_kernel");
    } else {
        switch (a.turb_model) {
        case ATJUP_TURB_K_EPSILON:
            closure_stage_kernel<ATJUP_TURB_K_EPSILON, TI, TO, TA, R><<<grid, block, 0, st>>>(a);
            break;
        case ATJUP_TURB_K_OMEGA:
            closure_stage_kernel<ATJUP_TURB_K_OMEGA, TI, TO, TA, R><<<grid, block, 0, st>>>(a);
            break;
        default:
            closure_stage_kernel<ATJUP_TURB_K_OMEGA_SST, TI, TO, TA, R><<<grid, block, 0, st>>>(a);
        }
        c->launches++;
        ATJUP_CHECK_LAUNCH("closure_stage_kernel");
    }
    return ATJUP_OK;
}

// species_stage_kernel of one RK stage (what = 0) or closure_stage_kernel (what = 1) on stream
// st; vin are the stage input's t, u, v, w (stage 0: the FP64 state; later stages: the stage
// buffers)
int launch_phys_stage(AtjupCtx* c, int stage, const void* const* vin, int what, cudaStream_t st) {
    const PhysStage a = stage_args(c, stage, vin);
    if (c->step_prec != ATJUP_PREC_MIXED) return launch_typed<double, double, double, double>(c, a, what, st);
    if (stage == 0) return launch_typed<double, float, float, float>(c, a, what, st);
    if (stage < 3) return launch_typed<float, float, float, float>(c, a, what, st);
    return launch_typed<float, double, float, float>(c, a, what, st);
}

}  // namespace atjup
