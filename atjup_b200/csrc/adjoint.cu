// Tangent-linear and adjoint of one RK4 step of the dry dynamics (t, u, v, w), linearised about
// the context's current state: RungeKuttaJup (RungeKutta_Jup_Turb.cpp:261-583) with the t, u, v,
// w right-hand sides of RHSJup (RHS_Jup_Turb.cpp:31-1457), the buoyancy level mean
// (computeBuoyancyRefLevel, RungeKutta_Jup_Turb.cpp:47-69) and the hydrostatic integral
// (computeHydrostaticPressure, 119-259). p_dyn, p_stat, rho_mix, wall_nue and the cell-hold means
// are inputs of the step, held fixed; the state itself is not advanced.
//
// Both directions first recompute the forward stages: the stage inputs X1, X2, X3 are kept in
// scratch (the forward stage kernel writes them with buffers of its own), and p_hydro and the
// level means, which the recompute overwrites, are saved and put back. Then
//   tangent-linear: the level mean's and the column integral's linearisations, and per stage one
//     thread per cell evaluating the linearised right-hand side from the forward stage input and
//     the perturbed one (7-point stencils), the RK bookkeeping carried along as in the forward
//     step;
//   adjoint: the stages in reverse, each a scatter: one thread per integrated cell forms the
//     adjoint of its right-hand sides (from the final update and the next stage's input),
//     transposes the cell's local Jacobian and adds it into the adjoints of the 7-point stencils
//     of t, u, v, w, of p_hydro's 5 points and of the level mean (FP64 atomic adds); then the
//     column integral and the level mean are transposed onto v, w and t.
// The stencils, the solid-face mirroring of p_hydro, the ring in phi and the integrated-cell mask
// are those of the forward kernel (rk4.cu), so the two directions are transposes of each other.
#include "ctx.cuh"

namespace atjup {
namespace {

enum : uint8_t { NB_S = 1, NB_IP = 2, NB_IM = 4, NB_JP = 8, NB_JM = 16, NB_KP = 32, NB_KM = 64,
                 NB_INT = 128 };

constexpr int LB_THREADS = 256;   // level-mean reduction block

struct LinConst {
    int im, jm, km, KP;
    double dt, dr;
    double inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
    double cor_phi_f, coeff_energy_p, to_nd, r_mix, rR, g, t_ref;
    double t_visc, inv_re, buoy_k, metric_on, cor_rad_on, Coriolis, pgrad_scale;
    int pgrad_wall, adiabatic, adiabatic_rho, hydro_split, use_hp;
};

LinConst lin_const(const AtjupCtx* c) {
    const AtjupParams& P = c->P;
    LinConst q{};
    q.im = P.im; q.jm = P.jm; q.km = P.km; q.KP = c->KP;
    q.dt = P.dt;
    q.dr = P.dr;
    q.inv_2dr = 1.0 / (2.0 * P.dr);
    q.inv_2dthe = 1.0 / (2.0 * P.dthe);
    q.inv_2dphi = 1.0 / (2.0 * P.dphi);
    q.inv_dr2 = 1.0 / (P.dr * P.dr);
    q.inv_dthe2 = 1.0 / (P.dthe * P.dthe);
    q.inv_dphi2 = 1.0 / (P.dphi * P.dphi);
    q.cor_phi_f = P.nd_cor * +2.0 * P.omega;
    q.coeff_energy_p = P.u_0 * P.u_0 / (P.cp_mix * P.t_ref);
    q.to_nd = 1.0 / P.p_dyn_to_bar;
    q.r_mix = P.r_mix;
    q.rR = P.r_mix * P.R_mix;
    q.g = P.g;
    q.t_ref = P.t_ref;
    q.t_visc = P.t_diff_scale / (P.re * P.pr);
    q.inv_re = 1.0 / P.re;
    q.buoy_k = -P.nd_buoy * P.buoy_scale * P.buoy_ramp * P.buoyancy;
    q.metric_on = P.metric_split ? 0.0 : 1.0;
    q.cor_rad_on = P.coriolis_split ? 0.0 : 1.0;
    q.Coriolis = P.Coriolis;
    q.pgrad_scale = P.pgrad_scale;
    q.pgrad_wall = P.pgrad_wall;
    q.adiabatic = P.adiabatic;
    q.adiabatic_rho = P.adiabatic_rho;
    q.hydro_split = P.hydro_split;
    q.use_hp = (P.hydro_split || P.metric_split) ? 1 : 0;
    return q;
}

struct LinPtrs {
    const double* X[4];        // forward stage input t, u, v, w
    const double* Y[4];        // time-level-n state
    const double *p_dyn, *p_stat, *rho, *wall_nue;
    const uint8_t* nb;
    const GeoIJ* geo;
};

// the 7-point stencil of one cell: centre, i +- 1, j +- 1, k +- 1 (ring over km - 1 meridians)
struct Nbr {
    size_t c, ip, im, jp, jm, kp, km;
};
__device__ __forceinline__ Nbr nbr_of(const LinConst& q, int i, int j, int k) {
    Nbr n;
    const size_t row = ((size_t)i * q.jm + j) * q.KP, plane = (size_t)q.jm * q.KP;
    n.c = row + k;
    n.ip = (i < q.im - 1) ? n.c + plane : n.c;
    n.im = (i > 0) ? n.c - plane : n.c;
    n.jp = (j < q.jm - 1) ? n.c + q.KP : n.c;
    n.jm = (j > 0) ? n.c - q.KP : n.c;
    n.kp = row + ((k >= q.km - 2) ? 0 : k + 1);
    n.km = row + ((k == 0) ? q.km - 2 : k - 1);
    return n;
}

// first and second centred differences of a field at a cell (RHS_Jup_Turb.cpp:180-254)
struct Der {
    double f0, d1r, d2r, d1t, d2t, d1p, d2p;
};
__device__ __forceinline__ Der der_of(const LinConst& q, const double* F, const Nbr& n) {
    Der d;
    d.f0 = F[n.c];
    const double fip = F[n.ip], fim = F[n.im], fjp = F[n.jp], fjm = F[n.jm];
    const double fkp = F[n.kp], fkm = F[n.km];
    d.d1r = (fip - fim) * q.inv_2dr;
    d.d2r = (fip - 2.0 * d.f0 + fim) * q.inv_dr2;
    d.d1t = (fjp - fjm) * q.inv_2dthe;
    d.d2t = (fjp - 2.0 * d.f0 + fjm) * q.inv_dthe2;
    d.d1p = (fkp - fkm) * q.inv_2dphi;
    d.d2p = (fkp - 2.0 * d.f0 + fkm) * q.inv_dphi2;
    return d;
}

// the frozen terms of a cell's right-hand sides that multiply the state: the pressure gradients
// of p_dyn with the solid-face mirroring, the adiabatic p_stat gradient, the viscosity and B of
// the buoyancy (g p_stat / (rR t0 t_ref)) over t0
struct Frozen {
    double dpdr, dpdthe, dpdphi, dpstatdr, visc, dbdt0;
    bool buoy;
};
__device__ __forceinline__ Frozen frozen_of(const LinConst& q, const LinPtrs& a, const Nbr& n,
                                            uint8_t nbm, double t0) {
    Frozen z;
    const bool wall = q.pgrad_wall;
    const double* P = a.p_dyn;
    const double pc = P[n.c];
    const double pip = (wall && (nbm & NB_IP)) ? pc : P[n.ip];
    const double pim = (wall && (nbm & NB_IM)) ? pc : P[n.im];
    const double pjp = (wall && (nbm & NB_JP)) ? pc : P[n.jp];
    const double pjm = (wall && (nbm & NB_JM)) ? pc : P[n.jm];
    const double pkp = (wall && (nbm & NB_KP)) ? pc : P[n.kp];
    const double pkm = (wall && (nbm & NB_KM)) ? pc : P[n.km];
    z.dpdr = (pip - pim) * q.inv_2dr;
    z.dpdthe = (pjp - pjm) * q.inv_2dthe;
    z.dpdphi = (pkp - pkm) * q.inv_2dphi;
    const double rho_l = a.rho[n.c];
    z.dpstatdr = 0.0;
    if (q.adiabatic) {
        z.dpstatdr = (a.p_stat[n.ip] - a.p_stat[n.im]) * q.inv_2dr * q.to_nd;
        if (q.adiabatic_rho && rho_l > 0.0 && isfinite(rho_l)) z.dpstatdr *= q.r_mix / rho_l;
    }
    z.visc = q.inv_re + a.wall_nue[n.c];
    z.buoy = !q.hydro_split && t0 > 0.0;
    z.dbdt0 = 0.0;
    if (z.buoy) {
        const double B = q.g * a.p_stat[n.c] / (q.rR * t0 * q.t_ref);
        z.dbdt0 = -B / t0;
    }
    return z;
}

// the six p_dyn neighbours of the pressure gradients, a solid face mirrored to the cell itself
// (RHS_Jup_Turb.cpp:119-130): i+, i-, j+, j-, k+, k-
__device__ __forceinline__ void p_nbrs(const LinConst& q, const Nbr& n, uint8_t nbm, size_t* o) {
    const bool wall = q.pgrad_wall;
    o[0] = (wall && (nbm & NB_IP)) ? n.c : n.ip;
    o[1] = (wall && (nbm & NB_IM)) ? n.c : n.im;
    o[2] = (wall && (nbm & NB_JP)) ? n.c : n.jp;
    o[3] = (wall && (nbm & NB_JM)) ? n.c : n.jm;
    o[4] = (wall && (nbm & NB_KP)) ? n.c : n.kp;
    o[5] = (wall && (nbm & NB_KM)) ? n.c : n.km;
}

// d(dpstatdr)/d(rho) / dpstatdr of the compression work with ATJUP_ADIABATIC_RHO: -1/rho where
// the forward divides by rho, else 0
__device__ __forceinline__ double dpstat_rho_factor(const LinConst& q, double rho_l) {
    return (q.adiabatic && q.adiabatic_rho && rho_l > 0.0 && isfinite(rho_l)) ? -1.0 / rho_l : 0.0;
}

// the mirrored p_hydro neighbours of the v and w equations: the cell itself at a solid face
__device__ __forceinline__ void ph_nbrs(const LinConst& q, const Nbr& n, uint8_t nbm, size_t& jp,
                                        size_t& jm, size_t& kp, size_t& km) {
    const bool wall = q.pgrad_wall;
    jp = (wall && (nbm & NB_JP)) ? n.c : n.jp;
    jm = (wall && (nbm & NB_JM)) ? n.c : n.jm;
    kp = (wall && (nbm & NB_KP)) ? n.c : n.kp;
    km = (wall && (nbm & NB_KM)) ? n.c : n.km;
}

// ---- tangent-linear stage: one thread per cell
// dX: the perturbed stage input; dY: the perturbation of the time-level-n state; dph: of p_hydro;
// db: of the level means; dacc: the accumulators; dXo: the next stage input (stage 3: the result)
struct TlArgs {
    LinPtrs a;
    const double* dX[4];
    const double* dY[4];
    double* dXo[4];
    double* dacc[4];
    const double* dph;
    const double* db;
    const double* dp;          // perturbation of p_dyn (null: held fixed)
    const double* drho;        // perturbation of rho_mix (null: held fixed)
    double* daux[3];           // stage 3: aux_u, aux_v, aux_w, written at integrated cells (null: none)
    int stage;
    double c_in, wgt;
};

__global__ void tl_stage_kernel(TlArgs A, LinConst q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    if (k >= q.km) return;
    const Nbr n = nbr_of(q, i, j, k);
    const uint8_t nbm = A.a.nb[n.c];
    if (!(nbm & NB_INT)) {      // the cell keeps its time-level-n value through the step
        for (int f = 0; f < 4; f++) A.dXo[f][n.c] = A.dY[f][n.c];
        return;
    }
    const GeoIJ& g = A.a.geo[(size_t)i * q.jm + j];
    const Der T = der_of(q, A.a.X[0], n), U = der_of(q, A.a.X[1], n);
    const Der V = der_of(q, A.a.X[2], n), W = der_of(q, A.a.X[3], n);
    const Der dT = der_of(q, A.dX[0], n), dU = der_of(q, A.dX[1], n);
    const Der dV = der_of(q, A.dX[2], n), dW = der_of(q, A.dX[3], n);
    const Frozen z = frozen_of(q, A.a, n, nbm, T.f0);
    const double u0 = U.f0, v0 = V.f0, w0 = W.f0;
    const double du0 = dU.f0, dv0 = dV.f0, dw0 = dW.f0;
    const double irm = g.inv_rm, irs = g.inv_rmsinthe, irm2 = g.inv_rm2, ci = g.costhe_inv_rm2sinthe;
    const double is2 = g.inv_rm2sinthe2, cot = g.cotanthe;

    const double d_pressure_t = q.coeff_energy_p *
        (du0 * (z.dpdr + z.dpstatdr) + dv0 * irm * z.dpdthe + dw0 * irs * z.dpdphi);
    const double d_transport_t = du0 * T.d1r + u0 * dT.d1r + dv0 * irm * T.d1t + v0 * irm * dT.d1t +
                                 dw0 * irs * T.d1p + w0 * irs * dT.d1p;
    const double d_transport_u = du0 * U.d1r + u0 * dU.d1r + dv0 * irm * U.d1t + v0 * irm * dU.d1t +
                                 dw0 * irs * U.d1p + w0 * irs * dU.d1p -
                                 q.metric_on * (2.0 * v0 * dv0 + 2.0 * w0 * dw0) * irm;
    const double d_transport_v = du0 * V.d1r + u0 * dV.d1r + dv0 * irm * V.d1t + v0 * irm * dV.d1t +
                                 dw0 * irs * V.d1p + w0 * irs * dV.d1p +
                                 (du0 * v0 + u0 * dv0 - 2.0 * w0 * dw0 * cot) * irm;
    const double d_transport_w = du0 * W.d1r + u0 * dW.d1r + dv0 * irm * W.d1t + v0 * irm * dW.d1t +
                                 dw0 * irs * W.d1p + w0 * irs * dW.d1p +
                                 (dw0 * u0 + w0 * du0 + (dv0 * w0 + v0 * dw0) * cot) * irm;
    const double two_irm = 2.0 * irm;
    const double d_diff_t = dT.d2r + dT.d1r * two_irm + dT.d2t * irm2 + dT.d1t * ci + dT.d2p * is2;
    const double d_diff_u = dU.d2r + 2.0 * du0 * irm2 + dU.d2t * irm2 + 4.0 * dU.d1r * irm +
                            dU.d1t * ci + dU.d2p * is2;
    const double d_diff_v = dV.d2r + dV.d1r * two_irm + dV.d2t * irm2 + dV.d1t * ci - g.v_metric * dv0 +
                            dV.d2p * is2 + 2.0 * dU.d1t * irm2 - dW.d1p * 2.0 * g.costhe * is2;
    const double d_diff_w = dW.d2r + dW.d1r * two_irm + dW.d2t * irm2 + dW.d1t * ci - g.v_metric * dw0 +
                            dW.d2p * is2 + 2.0 * dU.d1p * g.inv_rm2sinthe + dV.d1p * 2.0 * g.costhe * is2;
    double d_dph_the = 0.0, d_dph_phi = 0.0;
    if (q.use_hp) {
        size_t jp, jm, kp, km;
        ph_nbrs(q, n, nbm, jp, jm, kp, km);
        d_dph_the = (A.dph[jp] - A.dph[jm]) * q.inv_2dthe * irm;
        d_dph_phi = (A.dph[kp] - A.dph[km]) * q.inv_2dphi * irs;
    }
    const double d_buoy = z.buoy ? q.buoy_k * (z.dbdt0 * dT.f0 - A.db[i]) : 0.0;
    // the pressure gradients of a perturbed p_dyn and the compression work of a perturbed rho
    double ddpdr = 0.0, ddpdthe = 0.0, ddpdphi = 0.0, ddpstat = 0.0;
    if (A.dp) {
        size_t o[6];
        p_nbrs(q, n, nbm, o);
        ddpdr = (A.dp[o[0]] - A.dp[o[1]]) * q.inv_2dr;
        ddpdthe = (A.dp[o[2]] - A.dp[o[3]]) * q.inv_2dthe;
        ddpdphi = (A.dp[o[4]] - A.dp[o[5]]) * q.inv_2dphi;
    }
    if (A.drho) ddpstat = z.dpstatdr * dpstat_rho_factor(q, A.a.rho[n.c]) * A.drho[n.c];
    const double d_pressure_p = q.coeff_energy_p *
        (u0 * (ddpdr + ddpstat) + v0 * irm * ddpdthe + w0 * irs * ddpdphi);
    const double gp_u = q.pgrad_scale * ddpdr;
    const double gp_v = q.pgrad_scale * ddpdthe * irm;
    const double gp_w = q.pgrad_scale * ddpdphi * irs;

    const double dr_t = d_pressure_t + d_pressure_p - d_transport_t + d_diff_t * q.t_visc;
    const double dr_u = -gp_u + (q.hydro_split ? 0.0 : d_buoy) - d_transport_u + d_diff_u * z.visc -
                        q.cor_rad_on * q.Coriolis * g.cor_rad * dw0;
    const double dr_v = -gp_v - d_dph_the - d_transport_v + d_diff_v * z.visc -
                        q.Coriolis * g.cor_the * dw0;
    const double dr_w = -gp_w - d_dph_phi - d_transport_w + d_diff_w * z.visc -
                        q.Coriolis * q.cor_phi_f * (g.costhe * dv0 + g.sinthe_true * du0);
    const double drhs[4] = {dr_t, dr_u, dr_v, dr_w};
    if (A.stage == 3 && A.daux[0]) {   // aux = rhs + the p_dyn gradient term (rk4.cu)
        A.daux[0][n.c] = dr_u + gp_u;
        A.daux[1][n.c] = dr_v + gp_v;
        A.daux[2][n.c] = dr_w + gp_w;
    }
    for (int f = 0; f < 4; f++) {
        const double acc = (A.stage == 0) ? A.wgt * drhs[f] : A.dacc[f][n.c] + A.wgt * drhs[f];
        if (A.stage < 3) {
            A.dacc[f][n.c] = acc;
            A.dXo[f][n.c] = A.dY[f][n.c] + A.c_in * drhs[f];
        } else {
            A.dXo[f][n.c] = A.dY[f][n.c] + q.dt * acc * (1.0 / 6.0);
        }
    }
}

// ---- adjoint stage: one thread per integrated cell, scattering into lX (t, u, v, w), lph, lb
struct AdArgs {
    LinPtrs a;
    const double* lYn[4];      // adjoint of the step's result
    double* lXn[4];            // adjoint of the next stage input (stages 0-2); cleared here
    double* lX[4];             // adjoint of this stage's input (accumulated; zero on entry)
    double* lY[4];             // adjoint of the step's input (accumulated)
    double* lph;               // adjoint of p_hydro (accumulated)
    double* lb;                // adjoint of the level means (accumulated)
    double* lp;                // adjoint of p_dyn (accumulated; null: p_dyn held fixed)
    double* lrho;              // adjoint of rho_mix (accumulated; null: held fixed)
    double* laux[3];           // stage 3: adjoint of aux_u, aux_v, aux_w, read and cleared at the
                               // integrated cells (null: aux not an output)
    int stage;
    double c_in, wgt;
};

// the transposed differences of one field at one cell: the four i and j neighbours are added at
// once; the centre and the two phi neighbours are returned (cc, cp, cm) and combined across the
// warp below, where the phi neighbours are the adjacent lanes
__device__ __forceinline__ void scatter_field(const LinConst& q, double* L, const Nbr& n,
                                              double a0, double a1r, double a2r, double a1t,
                                              double a2t, double a1p, double a2p, double& cc,
                                              double& cp, double& cm) {
    atomicAdd(L + n.ip, a1r * q.inv_2dr + a2r * q.inv_dr2);
    atomicAdd(L + n.im, -a1r * q.inv_2dr + a2r * q.inv_dr2);
    atomicAdd(L + n.jp, a1t * q.inv_2dthe + a2t * q.inv_dthe2);
    atomicAdd(L + n.jm, -a1t * q.inv_2dthe + a2t * q.inv_dthe2);
    cp = a1p * q.inv_2dphi + a2p * q.inv_dphi2;
    cm = -a1p * q.inv_2dphi + a2p * q.inv_dphi2;
    cc = a0 - 2.0 * (a2r * q.inv_dr2 + a2t * q.inv_dthe2 + a2p * q.inv_dphi2);
}

__global__ void ad_stage_kernel(AdArgs A, LinConst q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    double lb_cell = 0.0;
    // per field: the adjoint added at the cell itself and at its phi+ and phi- neighbours
    double cc[4] = {0.0, 0.0, 0.0, 0.0}, cp[4] = {0.0, 0.0, 0.0, 0.0}, cm[4] = {0.0, 0.0, 0.0, 0.0};
    size_t at_c = 0, at_kp = 0, at_km = 0;
    if (k < q.km) {
        const Nbr n = nbr_of(q, i, j, k);
        const uint8_t nbm = A.a.nb[n.c];
        // every cell: the next stage input is Y + c_in rhs, so its adjoint (complete once the
        // next stage's scatter is done) adds to the input's; its buffer is then cleared for the
        // scatter of the stage below (stage 3 has none to read and only clears)
        double lxn[4] = {0.0, 0.0, 0.0, 0.0};
        for (int f = 0; f < 4; f++) {
            if (A.stage < 3) {
                lxn[f] = A.lXn[f][n.c];
                A.lY[f][n.c] += lxn[f];
            }
            A.lXn[f][n.c] = 0.0;
        }
        if (nbm & NB_INT) {
            // the adjoint of the cell's right-hand sides: from the final update (dt/6 wgt) and,
            // for stages 0-2, from the next stage input (c_in)
            double lr[4];
            for (int f = 0; f < 4; f++) lr[f] = q.dt * (1.0 / 6.0) * A.wgt * A.lYn[f][n.c] + A.c_in * lxn[f];
            // stage 3 also writes aux = rhs + the p_dyn gradient term of u, v, w: its adjoint adds
            // to the right-hand sides' adjoints everywhere but in the p_dyn gradients
            double lax = 0.0, lay = 0.0, law = 0.0;
            if (A.stage == 3 && A.laux[0]) {
                lax = A.laux[0][n.c]; lay = A.laux[1][n.c]; law = A.laux[2][n.c];
                A.laux[0][n.c] = 0.0; A.laux[1][n.c] = 0.0; A.laux[2][n.c] = 0.0;
            }
            const double at = lr[0], au = lr[1] + lax, av = lr[2] + lay, aw = lr[3] + law;
            const GeoIJ& g = A.a.geo[(size_t)i * q.jm + j];
            const Der T = der_of(q, A.a.X[0], n), U = der_of(q, A.a.X[1], n);
            const Der V = der_of(q, A.a.X[2], n), W = der_of(q, A.a.X[3], n);
            const Frozen z = frozen_of(q, A.a, n, nbm, T.f0);
            const double u0 = U.f0, v0 = V.f0, w0 = W.f0;
            const double irm = g.inv_rm, irs = g.inv_rmsinthe, irm2 = g.inv_rm2;
            const double ci = g.costhe_inv_rm2sinthe, is2 = g.inv_rm2sinthe2, cot = g.cotanthe;
            // adjoints of the centre values and of each field's six differences
            double At0 = 0.0, Au0 = 0.0, Av0 = 0.0, Aw0 = 0.0;
            double Tr1 = 0.0, Tr2 = 0.0, Tt1 = 0.0, Tt2 = 0.0, Tp1 = 0.0, Tp2 = 0.0;
            double Ur1 = 0.0, Ur2 = 0.0, Ut1 = 0.0, Ut2 = 0.0, Up1 = 0.0, Up2 = 0.0;
            double Vr1 = 0.0, Vr2 = 0.0, Vt1 = 0.0, Vt2 = 0.0, Vp1 = 0.0, Vp2 = 0.0;
            double Wr1 = 0.0, Wr2 = 0.0, Wt1 = 0.0, Wt2 = 0.0, Wp1 = 0.0, Wp2 = 0.0;
            // rhs_t = pressure_t - transport_t + diffusion_t t_visc
            Au0 += at * q.coeff_energy_p * (z.dpdr + z.dpstatdr);
            Av0 += at * q.coeff_energy_p * irm * z.dpdthe;
            Aw0 += at * q.coeff_energy_p * irs * z.dpdphi;
            Au0 -= at * T.d1r;  Tr1 -= at * u0;
            Av0 -= at * irm * T.d1t;  Tt1 -= at * v0 * irm;
            Aw0 -= at * irs * T.d1p;  Tp1 -= at * w0 * irs;
            {
                const double K = at * q.t_visc;
                Tr2 += K; Tr1 += K * 2.0 * irm; Tt2 += K * irm2; Tt1 += K * ci; Tp2 += K * is2;
            }
            // rhs_u = buoyancy - transport_u + diffusion_u visc - Coriolis_rad terms
            if (!q.hydro_split && z.buoy) {
                At0 += au * q.buoy_k * z.dbdt0;
                lb_cell -= au * q.buoy_k;
            }
            Au0 -= au * U.d1r;  Ur1 -= au * u0;
            Av0 -= au * irm * U.d1t;  Ut1 -= au * v0 * irm;
            Aw0 -= au * irs * U.d1p;  Up1 -= au * w0 * irs;
            Av0 += au * q.metric_on * 2.0 * v0 * irm;
            Aw0 += au * q.metric_on * 2.0 * w0 * irm;
            {
                const double Vs = au * z.visc;
                Ur2 += Vs; Au0 += Vs * 2.0 * irm2; Ut2 += Vs * irm2; Ur1 += Vs * 4.0 * irm;
                Ut1 += Vs * ci; Up2 += Vs * is2;
            }
            Aw0 -= au * q.cor_rad_on * q.Coriolis * g.cor_rad;
            // rhs_v = -dph_the - transport_v + diffusion_v visc - Coriolis_the
            double Ahjp = 0.0, Ahjm = 0.0, Ahkp = 0.0, Ahkm = 0.0;
            if (q.use_hp) {
                Ahjp -= av * q.inv_2dthe * irm;
                Ahjm += av * q.inv_2dthe * irm;
                Ahkp -= aw * q.inv_2dphi * irs;
                Ahkm += aw * q.inv_2dphi * irs;
            }
            Au0 -= av * (V.d1r + v0 * irm);  Vr1 -= av * u0;
            Av0 -= av * (irm * V.d1t + u0 * irm);  Vt1 -= av * v0 * irm;
            Aw0 -= av * (irs * V.d1p - 2.0 * w0 * cot * irm);  Vp1 -= av * w0 * irs;
            {
                const double Vs = av * z.visc;
                Vr2 += Vs; Vr1 += Vs * 2.0 * irm; Vt2 += Vs * irm2; Vt1 += Vs * ci;
                Av0 -= Vs * g.v_metric; Vp2 += Vs * is2; Ut1 += Vs * 2.0 * irm2;
                Wp1 -= Vs * 2.0 * g.costhe * is2;
            }
            Aw0 -= av * q.Coriolis * g.cor_the;
            // rhs_w = -dph_phi - transport_w + diffusion_w visc - Coriolis_phi
            Au0 -= aw * (W.d1r + w0 * irm);  Wr1 -= aw * u0;
            Av0 -= aw * (irm * W.d1t + w0 * cot * irm);  Wt1 -= aw * v0 * irm;
            Aw0 -= aw * (irs * W.d1p + u0 * irm + v0 * cot * irm);  Wp1 -= aw * w0 * irs;
            {
                const double Vs = aw * z.visc;
                Wr2 += Vs; Wr1 += Vs * 2.0 * irm; Wt2 += Vs * irm2; Wt1 += Vs * ci;
                Aw0 -= Vs * g.v_metric; Wp2 += Vs * is2; Up1 += Vs * 2.0 * g.inv_rm2sinthe;
                Vp1 += Vs * 2.0 * g.costhe * is2;
            }
            Av0 -= aw * q.Coriolis * q.cor_phi_f * g.costhe;
            Au0 -= aw * q.Coriolis * q.cor_phi_f * g.sinthe_true;

            if (A.lp) {
                // the p_dyn gradients: of the compression work (rhs_t) and of the momentum
                // equations (without the aux part, which cancels them)
                const double Gr = at * q.coeff_energy_p * u0 - q.pgrad_scale * lr[1];
                const double Gt = (at * q.coeff_energy_p * v0 - q.pgrad_scale * lr[2]) * irm;
                const double Gp = (at * q.coeff_energy_p * w0 - q.pgrad_scale * lr[3]) * irs;
                size_t o[6];
                p_nbrs(q, n, nbm, o);
                atomicAdd(A.lp + o[0], Gr * q.inv_2dr);
                atomicAdd(A.lp + o[1], -Gr * q.inv_2dr);
                atomicAdd(A.lp + o[2], Gt * q.inv_2dthe);
                atomicAdd(A.lp + o[3], -Gt * q.inv_2dthe);
                atomicAdd(A.lp + o[4], Gp * q.inv_2dphi);
                atomicAdd(A.lp + o[5], -Gp * q.inv_2dphi);
            }
            if (A.lrho)
                A.lrho[n.c] += at * q.coeff_energy_p * u0 * z.dpstatdr *
                               dpstat_rho_factor(q, A.a.rho[n.c]);
            scatter_field(q, A.lX[0], n, At0, Tr1, Tr2, Tt1, Tt2, Tp1, Tp2, cc[0], cp[0], cm[0]);
            scatter_field(q, A.lX[1], n, Au0, Ur1, Ur2, Ut1, Ut2, Up1, Up2, cc[1], cp[1], cm[1]);
            scatter_field(q, A.lX[2], n, Av0, Vr1, Vr2, Vt1, Vt2, Vp1, Vp2, cc[2], cp[2], cm[2]);
            scatter_field(q, A.lX[3], n, Aw0, Wr1, Wr2, Wt1, Wt2, Wp1, Wp2, cc[3], cp[3], cm[3]);
            if (q.use_hp) {
                size_t jp, jm, kp, km;
                ph_nbrs(q, n, nbm, jp, jm, kp, km);
                atomicAdd(A.lph + jp, Ahjp);
                atomicAdd(A.lph + jm, Ahjm);
                atomicAdd(A.lph + kp, Ahkp);
                atomicAdd(A.lph + km, Ahkm);
            }
        }
    }
    // The phi neighbours across the warp: a warp is 32 consecutive k of one (i, j) row, so lane l's
    // phi+ cell is lane l+1's and its phi- cell lane l-1's, unless the neighbour is across the
    // warp's edge or the ring's seam (k = km-2 -> 0, 0 -> km-2); those are added by atomics.
    {
        const int lane = threadIdx.x & 31;
        const bool own = k < q.km;
        if (own) {
            const size_t row = ((size_t)i * q.jm + j) * q.KP;
            at_c = row + k;
            at_kp = row + ((k >= q.km - 2) ? 0 : k + 1);
            at_km = row + ((k == 0) ? q.km - 2 : k - 1);
        }
        const bool send_p = lane == 31 || k >= q.km - 2;        // phi+ not taken by lane l+1
        const bool send_m = lane == 0 || k == 0;                 // phi- not taken by lane l-1
        const bool take_l = lane > 0 && k - 1 < q.km - 2;        // lane l-1's phi+ is this cell
        const bool take_r = lane < 31;                           // lane l+1's phi- is this cell
        for (int f = 0; f < 4; f++) {
            const double from_l = __shfl_up_sync(0xffffffffu, cp[f], 1);
            const double from_r = __shfl_down_sync(0xffffffffu, cm[f], 1);
            if (!own) continue;
            double tot = cc[f];
            if (take_l) tot += from_l;
            if (take_r) tot += from_r;
            if (tot != 0.0) atomicAdd(A.lX[f] + at_c, tot);
            if (send_p && cp[f] != 0.0) atomicAdd(A.lX[f] + at_kp, cp[f]);
            if (send_m && cm[f] != 0.0) atomicAdd(A.lX[f] + at_km, cm[f]);
        }
    }
    // the level mean's adjoint: a warp sum, one add per warp (a block lies in one level)
    for (int o = 16; o > 0; o >>= 1) lb_cell += __shfl_down_sync(0xffffffffu, lb_cell, o);
    if ((threadIdx.x & 31) == 0 && lb_cell != 0.0) atomicAdd(A.lb + i, lb_cell);
}

// lY += lX over every cell of the padded block
__global__ void add_kernel(double* __restrict__ y, const double* __restrict__ x, size_t n) {
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) y[c] += x[c];
}

// ---- level mean: per level i, W_i = sum of sin(the_j) over the cells the forward mean counts
// (fluid, t > 0, finite buoyancy) and, given dt, S_i = sum of sin(the_j) d(b)/dt dt / W_i, the
// perturbation of the level mean. Two fixed-order levels (deterministic): LB_PARTS blocks per
// level over interleaved rows, then one thread per level
constexpr int LB_PARTS = 16;

__global__ void __launch_bounds__(LB_THREADS)
lin_level_partial(const double* __restrict__ t, const double* __restrict__ dt,
                  const double* __restrict__ p_stat, const uint8_t* __restrict__ solid,
                  const double* __restrict__ sin_the, double* __restrict__ part, int jm, int km,
                  int KP, double g, double rR, double t_ref) {
    const int i = blockIdx.y, b = blockIdx.x;
    double s = 0.0, ws = 0.0;
    for (int j = b; j < jm; j += LB_PARTS) {
        const double wgt = sin_the[j];
        const size_t row = ((size_t)i * jm + j) * KP;
        for (int k = threadIdx.x; k < km; k += LB_THREADS) {
            if (solid[row + k]) continue;
            const double tt = t[row + k];
            if (!(tt > 0.0)) continue;
            const double bb = g * p_stat[row + k] / (rR * tt * t_ref);
            if (!isfinite(bb)) continue;
            ws += wgt;
            if (dt) s += wgt * (-bb / tt) * dt[row + k];
        }
    }
    __shared__ double sh_s[LB_THREADS / 32], sh_w[LB_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        ws += __shfl_down_sync(0xffffffffu, ws, o);
    }
    if ((threadIdx.x & 31) == 0) { sh_s[threadIdx.x >> 5] = s; sh_w[threadIdx.x >> 5] = ws; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0, tw = 0.0;
        for (int q = 0; q < LB_THREADS / 32; q++) { ts += sh_s[q]; tw += sh_w[q]; }
        part[(i * LB_PARTS + b) * 2 + 0] = ts;
        part[(i * LB_PARTS + b) * 2 + 1] = tw;
    }
}

__global__ void lin_level_final(const double* __restrict__ part, double* __restrict__ W,
                                double* __restrict__ S, int im) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= im) return;
    double ts = 0.0, tw = 0.0;
    for (int b = 0; b < LB_PARTS; b++) {
        ts += part[(i * LB_PARTS + b) * 2 + 0];
        tw += part[(i * LB_PARTS + b) * 2 + 1];
    }
    W[i] = tw;
    S[i] = (tw > 0.0) ? ts / tw : 0.0;
}

// the level mean's transpose: lt += lb_i sin(the_j) / W_i d(b)/dt over the counted cells
__global__ void ad_level_kernel(const double* __restrict__ t, const double* __restrict__ p_stat,
                                const uint8_t* __restrict__ solid,
                                const double* __restrict__ sin_the, const double* __restrict__ W,
                                const double* __restrict__ lb, double* __restrict__ lt, int jm,
                                int km, int KP, double g, double rR, double t_ref) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    if (k >= km || !(W[i] > 0.0)) return;
    const size_t c = ((size_t)i * jm + j) * KP + k;
    if (solid[c]) return;
    const double tt = t[c];
    if (!(tt > 0.0)) return;
    const double bb = g * p_stat[c] / (rR * tt * t_ref);
    if (!isfinite(bb)) return;
    lt[c] += lb[i] * sin_the[j] / W[i] * (-bb / tt);
}

// ---- hydrostatic integral (the forward's metric/Coriolis form), one thread per column
__device__ __forceinline__ bool column_run(const uint8_t* solid, size_t base, size_t plane, int im,
                                           int& i0, int& i1) {
    i0 = 0;
    while (i0 < im && solid[base + i0 * plane]) i0++;
    if (i0 >= im) return false;
    i1 = i0;
    while (i1 + 1 < im && !solid[base + (i1 + 1) * plane]) i1++;
    return true;
}

__global__ void tl_hydro_kernel(const double* __restrict__ v, const double* __restrict__ w,
                                const double* __restrict__ dv, const double* __restrict__ dw,
                                const uint8_t* __restrict__ solid, const double* __restrict__ rad,
                                const double* __restrict__ cor_col, double* __restrict__ dph,
                                int im, int jm, int km, int KP, double dr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (k >= km) return;
    const size_t plane = (size_t)jm * KP, base = (size_t)j * KP + k;
    for (int i = 0; i < im; i++) dph[base + i * plane] = 0.0;
    int i0, i1;
    if (!column_run(solid, base, plane, im, i0, i1)) return;
    const double cor = cor_col[j];
    double acc = 0.0, fprev = 0.0;
    for (int i = i0; i <= i1; i++) {
        const size_t c = base + i * plane;
        const double f = (2.0 * v[c] * dv[c] + 2.0 * w[c] * dw[c]) / rad[i] + cor * dw[c];
        if (i > i0) acc = acc + 0.5 * (fprev + f) * dr;
        fprev = f;
        dph[c] = acc;
    }
}

__global__ void ad_hydro_kernel(const double* __restrict__ v, const double* __restrict__ w,
                                const double* __restrict__ lph, const uint8_t* __restrict__ solid,
                                const double* __restrict__ rad, const double* __restrict__ cor_col,
                                double* __restrict__ lv, double* __restrict__ lw, int im, int jm,
                                int km, int KP, double dr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (k >= km) return;
    const size_t plane = (size_t)jm * KP, base = (size_t)j * KP + k;
    int i0, i1;
    if (!column_run(solid, base, plane, im, i0, i1)) return;
    const double cor = cor_col[j];
    double L = 0.0, carry = 0.0;     // carry: the adjoint of f_i from the increment of acc_{i+1}
    for (int i = i1; i >= i0; i--) {
        const size_t c = base + i * plane;
        L += lph[c];                  // the adjoint of acc_i (acc_{i+1} = acc_i + ...)
        double lf = carry;
        carry = 0.0;
        if (i > i0) {
            lf += 0.5 * dr * L;
            carry = 0.5 * dr * L;
        }
        lv[c] += lf * 2.0 * v[c] / rad[i];
        lw[c] += lf * (2.0 * w[c] / rad[i] + cor);
    }
}

// ---- orchestration
struct Lin {
    double* S[3][4];     // forward stage inputs X1, X2, X3
    double* A[2][4];     // ping-pong: tangent stage inputs, or adjoints of stage inputs
    double* B[4];        // tangent accumulators, or the adjoint of the step's result
    double* O[4];        // tangent result
    double* ph;          // tangent or adjoint of p_hydro
    double* ph_save;     // the context's p_hydro, put back after the recompute
    double* lv;          // [4 * im]: W, the level means' tangent or adjoint, the saved means
    double* part;        // [2 * LB_PARTS * im]: partial sums of the level means
};

int lin_setup(AtjupCtx* c, Lin& L) {
    const AtjupParams& P = c->P;
    if (c->phys_on || P.has_nue || P.has_heating) {
        set_error("rk4 tangent-linear/adjoint: the dry dynamics only (no physics block, nue or heating)");
        return ATJUP_ERR_UNSUPPORTED;
    }
    if (c->step_prec != ATJUP_PREC_FP64) {
        set_error("rk4 tangent-linear/adjoint: FP64 step only");
        return ATJUP_ERR_UNSUPPORTED;
    }
    if (!P.metric_split || P.hydro_split) {
        set_error("rk4 tangent-linear/adjoint: only the ATJUP_METRIC_SPLIT=1, ATJUP_HYDRO_SPLIT=0 form");
        return ATJUP_ERR_UNSUPPORTED;
    }
    const size_t NF = 30;
    if (!c->lin) {
        ATJUP_CUDA(cudaMalloc(&c->lin, sizeof(double) * (NF * c->NP + (4 + 2 * LB_PARTS) * (size_t)P.im)));
    }
    double* p = c->lin;
    for (int s = 0; s < 3; s++) for (int f = 0; f < 4; f++) { L.S[s][f] = p; p += c->NP; }
    for (int s = 0; s < 2; s++) for (int f = 0; f < 4; f++) { L.A[s][f] = p; p += c->NP; }
    for (int f = 0; f < 4; f++) { L.B[f] = p; p += c->NP; }
    for (int f = 0; f < 4; f++) { L.O[f] = p; p += c->NP; }
    L.ph = p; p += c->NP;
    L.ph_save = p; p += c->NP;
    L.lv = p;
    L.part = p + 4 * (size_t)P.im;
    return ATJUP_OK;
}

// the forward stages 0-2 into L.S (unless `stages` holds them), with p_hydro and the level means
// of this state
int lin_forward(AtjupCtx* c, Lin& L, const double* const* stages = nullptr) {
    const AtjupParams& P = c->P;
    double* Y[4] = {c->f[ATJUP_F_T], c->f[ATJUP_F_U], c->f[ATJUP_F_V], c->f[ATJUP_F_W]};
    ATJUP_CUDA(cudaMemcpyAsync(L.ph_save, c->f[ATJUP_F_P_HYDRO], sizeof(double) * c->NP,
                               cudaMemcpyDeviceToDevice, c->stream));
    ATJUP_CUDA(cudaMemcpyAsync(L.lv + 3 * P.im, c->buoy_ref, sizeof(double) * P.im,
                               cudaMemcpyDeviceToDevice, c->stream));
    int rc;
    if ((rc = launch_buoy_ref(c, Y[0]))) return rc;
    if ((rc = launch_hydrostatic(c, Y[2], Y[3]))) return rc;
    if (stages) {
        for (int s = 0; s < 3; s++)
            for (int f = 0; f < 4; f++) L.S[s][f] = const_cast<double*>(stages[4 * s + f]);
        return ATJUP_OK;
    }
    for (int s = 0; s < 3; s++) {
        const void* in[4];
        void* out[4];
        for (int f = 0; f < 4; f++) {
            in[f] = (s == 0) ? (const void*)Y[f] : (const void*)L.S[s - 1][f];
            out[f] = L.S[s][f];
        }
        const void* x1[4] = {L.S[0][0], L.S[0][1], L.S[0][2], L.S[0][3]};
        if ((rc = launch_rk_stage(c, s, in, out, x1))) return rc;
    }
    return ATJUP_OK;
}

int lin_restore(AtjupCtx* c, Lin& L) {
    ATJUP_CUDA(cudaMemcpyAsync(c->f[ATJUP_F_P_HYDRO], L.ph_save, sizeof(double) * c->NP,
                               cudaMemcpyDeviceToDevice, c->stream));
    ATJUP_CUDA(cudaMemcpyAsync(c->buoy_ref, L.lv + 3 * c->P.im, sizeof(double) * c->P.im,
                               cudaMemcpyDeviceToDevice, c->stream));
    return ATJUP_OK;
}

LinPtrs lin_ptrs(AtjupCtx* c, const Lin& L, int stage) {
    LinPtrs a{};
    for (int f = 0; f < 4; f++) {
        a.Y[f] = c->f[ATJUP_F_T + f];
        a.X[f] = (stage == 0) ? c->f[ATJUP_F_T + f] : L.S[stage - 1][f];
    }
    a.p_dyn = c->f[ATJUP_F_P_DYN];
    a.p_stat = c->f[ATJUP_F_P_STAT];
    a.rho = c->f[ATJUP_F_RHO_MIX];
    a.wall_nue = c->f[ATJUP_F_WALL_NUE];
    a.nb = c->nbflags;
    a.geo = c->geo;
    return a;
}

double stage_c_in(const AtjupParams& P, int s) {
    return (s == 0 || s == 1) ? 0.5 * P.dt : (s == 2 ? P.dt : 0.0);
}
double stage_wgt(int s) { return (s == 0 || s == 3) ? 1.0 : 2.0; }

}  // namespace
}  // namespace atjup

using namespace atjup;

extern "C" {

int atjup_gpu_rk4_tlm(AtjupCtx* c, double* const d[4]) {
    if (!c || !d || !d[0] || !d[1] || !d[2] || !d[3]) { set_error("rk4_tlm: null argument"); return ATJUP_ERR_ARG; }
    if (!c->grid_set) { set_error("rk4_tlm: atjup_gpu_set_grid was not called"); return ATJUP_ERR_ARG; }
    return rk4_tlm_ext(c, d, nullptr, nullptr, nullptr);
}

int atjup_gpu_rk4_adjoint(AtjupCtx* c, double* const a[4]) {
    if (!c || !a || !a[0] || !a[1] || !a[2] || !a[3]) { set_error("rk4_adjoint: null argument"); return ATJUP_ERR_ARG; }
    if (!c->grid_set) { set_error("rk4_adjoint: atjup_gpu_set_grid was not called"); return ATJUP_ERR_ARG; }
    return rk4_adjoint_ext(c, a, nullptr, nullptr, nullptr);
}

}  // extern "C"

namespace atjup {

int rk4_tlm_ext(AtjupCtx* c, double* const d[4], const double* dp, const double* drho,
                double* const daux[3]) {
    Lin L;
    int rc;
    if ((rc = lin_setup(c, L))) return rc;
    if ((rc = lin_forward(c, L))) return rc;
    const AtjupParams& P = c->P;
    const LinConst q = lin_const(c);
    double* W = L.lv;
    double* db = L.lv + P.im;
    lin_level_partial<<<dim3(LB_PARTS, P.im), LB_THREADS, 0, c->stream>>>(
        c->f[ATJUP_F_T], d[0], c->f[ATJUP_F_P_STAT], c->solid, c->sin_the, L.part, P.jm, P.km,
        c->KP, q.g, q.rR, q.t_ref);
    lin_level_final<<<(P.im + 63) / 64, 64, 0, c->stream>>>(L.part, W, db, P.im);
    c->launches++;
    tl_hydro_kernel<<<dim3((P.km + 127) / 128, P.jm), 128, 0, c->stream>>>(
        c->f[ATJUP_F_V], c->f[ATJUP_F_W], d[2], d[3], c->solid, c->rad, c->cor_col, L.ph, P.im,
        P.jm, P.km, c->KP, P.dr);
    c->launches += 2;
    ATJUP_CHECK_LAUNCH("rk4_tlm: level mean / hydrostatic");
    const dim3 grid((P.km + 127) / 128, P.jm, P.im);
    // the result's lanes k >= km are never written by the stage kernel: zero them
    for (int f = 0; f < 4; f++) ATJUP_CUDA(cudaMemsetAsync(L.O[f], 0, sizeof(double) * c->NP, c->stream));
    for (int s = 0; s < 4; s++) {
        TlArgs A{};
        A.a = lin_ptrs(c, L, s);
        for (int f = 0; f < 4; f++) {
            A.dX[f] = (s == 0) ? d[f] : L.A[(s - 1) & 1][f];
            A.dY[f] = d[f];
            A.dXo[f] = (s < 3) ? L.A[s & 1][f] : L.O[f];
            A.dacc[f] = L.B[f];
        }
        A.dph = L.ph;
        A.db = db;
        A.dp = dp;
        A.drho = drho;
        for (int f = 0; f < 3; f++) A.daux[f] = daux ? daux[f] : nullptr;
        A.stage = s;
        A.c_in = stage_c_in(P, s);
        A.wgt = stage_wgt(s);
        tl_stage_kernel<<<grid, 128, 0, c->stream>>>(A, q);
        c->launches++;
        ATJUP_CHECK_LAUNCH("rk4_tlm: stage");
    }
    for (int f = 0; f < 4; f++)
        ATJUP_CUDA(cudaMemcpyAsync(d[f], L.O[f], sizeof(double) * c->NP, cudaMemcpyDeviceToDevice,
                                   c->stream));
    return lin_restore(c, L);
}

int rk4_adjoint_ext(AtjupCtx* c, double* const a[4], double* lp, double* lrho,
                    double* const laux[3], const double* const* stages) {
    Lin L;
    int rc;
    if ((rc = lin_setup(c, L))) return rc;
    if ((rc = lin_forward(c, L, stages))) return rc;
    const AtjupParams& P = c->P;
    const LinConst q = lin_const(c);
    const size_t bytes = sizeof(double) * c->NP;
    // the adjoint of the result, kept: every stage reads it; a[] accumulates the adjoint of Y
    for (int f = 0; f < 4; f++)
        ATJUP_CUDA(cudaMemcpyAsync(L.B[f], a[f], bytes, cudaMemcpyDeviceToDevice, c->stream));
    double* W = L.lv;
    double* lb = L.lv + P.im;
    ATJUP_CUDA(cudaMemsetAsync(L.ph, 0, bytes, c->stream));
    ATJUP_CUDA(cudaMemsetAsync(lb, 0, sizeof(double) * P.im, c->stream));
    const dim3 grid((P.km + 127) / 128, P.jm, P.im);
    const unsigned nblk = (unsigned)((c->NP + 255) / 256);
    // stage 3 scatters into A[1]; every later stage's target was cleared by the stage before it
    for (int f = 0; f < 4; f++) ATJUP_CUDA(cudaMemsetAsync(L.A[1][f], 0, bytes, c->stream));
    for (int s = 3; s >= 0; s--) {
        double* const* cur = L.A[s & 1];
        double* const* nxt = L.A[(s + 1) & 1];
        AdArgs A{};
        A.a = lin_ptrs(c, L, s);
        for (int f = 0; f < 4; f++) {
            A.lYn[f] = L.B[f];
            A.lXn[f] = nxt[f];
            A.lX[f] = cur[f];
            A.lY[f] = a[f];
        }
        A.lph = L.ph;
        A.lb = lb;
        A.lp = lp;
        A.lrho = lrho;
        for (int f = 0; f < 3; f++) A.laux[f] = laux ? laux[f] : nullptr;
        A.stage = s;
        A.c_in = stage_c_in(P, s);
        A.wgt = stage_wgt(s);
        ad_stage_kernel<<<grid, 128, 0, c->stream>>>(A, q);
        c->launches++;
        ATJUP_CHECK_LAUNCH("rk4_adjoint: stage");
    }
    // the adjoint of stage 0's input, which is Y itself
    for (int f = 0; f < 4; f++) add_kernel<<<nblk, 256, 0, c->stream>>>(a[f], L.A[0][f], c->NP);
    c->launches += 4;
    // the column integral onto v, w and the level mean onto t
    ad_hydro_kernel<<<dim3((P.km + 127) / 128, P.jm), 128, 0, c->stream>>>(
        c->f[ATJUP_F_V], c->f[ATJUP_F_W], L.ph, c->solid, c->rad, c->cor_col, a[2], a[3], P.im,
        P.jm, P.km, c->KP, P.dr);
    lin_level_partial<<<dim3(LB_PARTS, P.im), LB_THREADS, 0, c->stream>>>(
        c->f[ATJUP_F_T], nullptr, c->f[ATJUP_F_P_STAT], c->solid, c->sin_the, L.part, P.jm, P.km,
        c->KP, q.g, q.rR, q.t_ref);
    lin_level_final<<<(P.im + 63) / 64, 64, 0, c->stream>>>(L.part, W, L.lv + 2 * P.im, P.im);
    c->launches++;
    ad_level_kernel<<<grid, 128, 0, c->stream>>>(c->f[ATJUP_F_T], c->f[ATJUP_F_P_STAT], c->solid,
                                                 c->sin_the, W, lb, a[0], P.jm, P.km, c->KP, q.g,
                                                 q.rR, q.t_ref);
    c->launches += 3;
    ATJUP_CHECK_LAUNCH("rk4_adjoint: hydrostatic / level mean");
    return lin_restore(c, L);
}

}  // namespace atjup
