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
    // stage input velocities
    const double *u, *v, *w;
    // scalars: stage input, next stage input (stage 3: the live field), time-level n,
    // accumulator, live field (for the non-integrated copy)
    const double* q_in[ATJUP_S_COUNT + 2];
    double* q_out[ATJUP_S_COUNT + 2];
    const double* q_n[ATJUP_S_COUNT + 2];
    double* acc[ATJUP_S_COUNT + 2];
    const double* q_live[ATJUP_S_COUNT + 2];
    // frozen inputs
    const double* sprec[9];
    const double *mf_h2s, *mf_nh3, *mf_nh4sh, *fluxlim;
    const double *nue, *rho_mix;
    const double* t;                   // stage input temperature
    const double* vel_star;            // [jm][KP]
    const float* layer_h;              // [im]
    const int32_t* topo;               // [jm * km]
    // closure outputs
    double *prod, *tke_source, *dis_source;
    const uint8_t* flags;
    const GeoIJ* geo;
    int im, jm, km, KP, stage;
    double c_in, wgt, dt, one_sixth;
    double inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
    double coef[ATJUP_S_COUNT];        // species_diff_scale / (sc re)
    double precip_coupling, chemical_reaction, turb_coupling;
    double stokes_pre, rg_nh4sh, mue_mix;  // (2/9) r_p r_p, computed in the reference's order
    double inv_re, L_m, u_0, t_ref, g, cp_mix, nue_max, tke_max_nd, re_turb, turb_buoy_prt;
    int has_nue, turb_model, turb_buoy;
};

__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }   // std::max
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }   // std::min

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

__device__ __forceinline__ Cell cell_of(const PhysStage& a, int i, int j, int k) {
    Cell x;
    const size_t row = ((size_t)i * a.jm + j) * a.KP;
    const int ke = (k >= a.km - 2) ? 0 : k + 1, kw = (k == 0) ? a.km - 2 : k - 1;
    x.c = row + k;
    x.cip = x.c + (size_t)a.jm * a.KP;
    x.cim = x.c - (size_t)a.jm * a.KP;
    x.cjp = x.c + a.KP;
    x.cjm = x.c - a.KP;
    x.ckp = row + ke;
    x.ckm = row + kw;
    return x;
}

// RK bookkeeping of one scalar at an integrated cell (RungeKutta_Jup_Turb.cpp:425-490, 493-568)
__device__ __forceinline__ void rk_update(const PhysStage& a, int s, size_t c, double rhs) {
    const double acc = (a.stage == 0) ? a.wgt * rhs : a.acc[s][c] + a.wgt * rhs;
    const double qn = a.q_n[s][c];
    if (a.stage < 3) {
        a.acc[s][c] = acc;
        double x = qn + a.c_in * rhs;
        if (s == ATJUP_S_COUNT) x = safe_clamp(x, 0.0, a.tke_max_nd);          // k*
        else if (s == ATJUP_S_COUNT + 1) x = dmax(1.0e-10, x);                 // omega*
        a.q_out[s][c] = x;
    } else {
        double x = qn + a.dt * acc * a.one_sixth;
        if (s == ATJUP_S_COUNT) x = safe_clamp(x, 0.0, a.tke_max_nd);
        else if (s == ATJUP_S_COUNT + 1) x = dmax(1.0e-10, x);
        else if (s == ATJUP_S_NH4SH) x = (x < 0.0) ? 0.0 : x;                  // keeps NaN, -0
        else x = dmax(0.0, x);
        a.q_out[s][c] = x;
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

// One thread per (cell, species): blockIdx.z = i * ATJUP_S_COUNT + species, so the eleven species
// blocks of one radial plane run back to back and the plane's u, v, w, nue come from DRAM once and
// from L2 for the other ten; each species' stencil is its own coalesced stream.
// blockIdx.y * blockDim.y + threadIdx.y = j, blockIdx.x * blockDim.x + threadIdx.x = k.
__global__ void __launch_bounds__(256) species_stage_kernel(PhysStage a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z / ATJUP_S_COUNT;
    const int s = blockIdx.z - i * ATJUP_S_COUNT;
    if (k >= a.km || j >= a.jm) return;
    // Every load is issued before the integrated-cell test (one memory round trip, not two):
    // the neighbour addresses are clamped into the block, so the boundary cells that the test
    // then sends to the copy below read only their own cell.
    const size_t plane = (size_t)a.jm * a.KP, row = ((size_t)i * a.jm + j) * a.KP;
    const size_t c = row + k;
    const int ke = (k >= a.km - 2) ? 0 : k + 1, kw = (k == 0) ? a.km - 2 : k - 1;
    const size_t cip = (i < a.im - 1) ? c + plane : c, cim = (i > 0) ? c - plane : c;
    const size_t cjp = (j < a.jm - 1) ? c + a.KP : c, cjm = (j > 0) ? c - a.KP : c;
    const size_t ckp = row + ke, ckm = row + kw;
    const double* F = a.q_in[s];
    const uint8_t fl = a.flags[c];
    const double f0 = F[c], fip = F[cip], fim = F[cim], fjp = F[cjp], fjm = F[cjm];
    const double fkp = F[ckp], fkm = F[ckm];
    const double u0 = a.u[c], v0 = a.v[c], w0 = a.w[c];
    const double nv = a.has_nue ? a.nue[c] : 0.0;
    const double qn = a.q_n[s][c];
    const double acc_in = (a.stage == 0) ? 0.0 : a.acc[s][c];
    double src0, src1 = 0.0, src2 = 0.0;
    if (s == ATJUP_S_H2S) {
        src0 = a.mf_h2s[c];
    } else if (s == ATJUP_S_NH3) {
        src0 = a.mf_nh3[c];
        src1 = a.sprec[3][c];
    } else if (s == ATJUP_S_NH4SH) {
        src0 = a.fluxlim[c];
        src1 = a.mf_nh4sh[c];
        src2 = a.rho_mix[c];
    } else {
        src0 = a.sprec[precip_slot(s)][c];
    }
    if (!(fl & NB_INT)) {
        if (a.stage < 3) a.q_out[s][c] = a.q_live[s][c];
        return;
    }
    const GeoIJ& g = a.geo[(size_t)i * a.jm + j];
    const double v_invrm = v0 * g.inv_rm;
    const double w_invrs = w0 * g.inv_rmsinthe;
    const double two_inv_rm = 2.0 * g.inv_rm;
    double nue_t = 0.0;
    if (a.has_nue && a.turb_coupling != 0.0 && isfinite(nv)) nue_t = a.turb_coupling * dmax(0.0, nv);
    const double nue_t_s = nue_t / 0.9;
    const double d1r = (fip - fim) * a.inv_2dr;
    const double d2r = (fip - 2.0 * f0 + fim) * a.inv_dr2;
    const double d1t = (fjp - fjm) * a.inv_2dthe;
    const double d2t = (fjp - 2.0 * f0 + fjm) * a.inv_dthe2;
    const double d1p = (fkp - fkm) * a.inv_2dphi;
    const double d2p = (fkp - 2.0 * f0 + fkm) * a.inv_dphi2;
    const double transport = u0 * d1r + v_invrm * d1t + w_invrs * d1p;
    const double diffusion = d2r + d1r * two_inv_rm + d2t * g.inv_rm2 +
                             d1t * g.costhe_inv_rm2sinthe + d2p * g.inv_rm2sinthe2;
    const double coef = a.coef[s] + nue_t_s;
    double r;
    if (s == ATJUP_S_H2S) {
        r = -transport + diffusion * coef + a.chemical_reaction * src0;
    } else if (s == ATJUP_S_NH3) {
        r = -transport + diffusion * coef + a.chemical_reaction * src0 + a.precip_coupling * src1;
    } else if (s == ATJUP_S_NH4SH) {
        const double v_stokes = a.stokes_pre * (a.rg_nh4sh - src2) * a.g / a.mue_mix;
        r = -transport + src0 + diffusion * coef + a.chemical_reaction * src1 +
            (v_stokes / a.u_0) * d1r;
    } else {
        r = -transport + diffusion * coef + a.precip_coupling * src0;
    }
    // RK bookkeeping (RungeKutta_Jup_Turb.cpp:425-490, 493-568), the accumulator read above
    const double accv = (a.stage == 0) ? a.wgt * r : acc_in + a.wgt * r;
    if (a.stage < 3) {
        a.acc[s][c] = accv;
        a.q_out[s][c] = qn + a.c_in * r;
    } else {
        const double x = qn + a.dt * accv * a.one_sixth;
        a.q_out[s][c] = (s == ATJUP_S_NH4SH) ? ((x < 0.0) ? 0.0 : x) : dmax(0.0, x);
    }
}

// k*, omega*: transport, diffusion with the model's coefficients, and the closure sources
// one instantiation per closure model, so that each holds the registers of its own branch only
template <int MODEL>
__global__ void __launch_bounds__(256) closure_stage_kernel(PhysStage a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= a.km || j >= a.jm) return;
    const int ST = ATJUP_S_COUNT, SD = ATJUP_S_COUNT + 1;
    // Every load is issued before the integrated-cell test (one memory round trip): the
    // neighbour addresses are clamped into the block, so boundary cells read only their own
    // cell before the test sends them to the copy below.
    Cell x = cell_of(a, i, j, k);
    if (i == a.im - 1) x.cip = x.c;
    if (i == 0) x.cim = x.c;
    if (j == a.jm - 1) x.cjp = x.c;
    if (j == 0) x.cjm = x.c;
    const uint8_t fl = a.flags[x.c];
    const double* TK = a.q_in[ST];
    const double* DS = a.q_in[SD];
    const double tk0 = TK[x.c], ds0 = DS[x.c];
    const double tip_ = TK[x.cip], tim_ = TK[x.cim], tjp_ = TK[x.cjp], tjm_ = TK[x.cjm];
    const double tkp_ = TK[x.ckp], tkm_ = TK[x.ckm];
    const double dip_ = DS[x.cip], dim_ = DS[x.cim], djp_ = DS[x.cjp], djm_ = DS[x.cjm];
    const double dkp_ = DS[x.ckp], dkm_ = DS[x.ckm];
    const double u0 = a.u[x.c], v0 = a.v[x.c], w0 = a.w[x.c];
    const double uip = a.u[x.cip], uim = a.u[x.cim], vip = a.v[x.cip], vim = a.v[x.cim];
    const double wip = a.w[x.cip], wim = a.w[x.cim];
    const double ujp = a.u[x.cjp], ujm = a.u[x.cjm], vjp = a.v[x.cjp], vjm = a.v[x.cjm];
    const double wjp = a.w[x.cjp], wjm = a.w[x.cjm];
    const double ukp = a.u[x.ckp], ukm = a.u[x.ckm], vkp = a.v[x.ckp], vkm = a.v[x.ckm];
    const double wkp = a.w[x.ckp], wkm = a.w[x.ckm];
    const double nv = a.nue[x.c];
    const int32_t topo = a.topo[(size_t)j * a.km + k];
    if (!(fl & NB_INT)) {
        if (a.stage < 3) {
            a.q_out[ST][x.c] = a.q_live[ST][x.c];
            a.q_out[SD][x.c] = a.q_live[SD][x.c];
        }
        return;
    }
    const GeoIJ& g = a.geo[(size_t)i * a.jm + j];
    // the solid-face mirror (RHS_Jup_Turb.cpp:257-303): a solid neighbour reads as the cell
    const double tip = (fl & NB_IP) ? tk0 : tip_, tim = (fl & NB_IM) ? tk0 : tim_;
    const double tjp = (fl & NB_JP) ? tk0 : tjp_, tjm = (fl & NB_JM) ? tk0 : tjm_;
    const double tkp = (fl & NB_KP) ? tk0 : tkp_, tkm = (fl & NB_KM) ? tk0 : tkm_;
    const double dip = (fl & NB_IP) ? ds0 : dip_, dim = (fl & NB_IM) ? ds0 : dim_;
    const double djp = (fl & NB_JP) ? ds0 : djp_, djm = (fl & NB_JM) ? ds0 : djm_;
    const double dkp = (fl & NB_KP) ? ds0 : dkp_, dkm = (fl & NB_KM) ? ds0 : dkm_;
    const double dtkedr = (tip - tim) * a.inv_2dr, d2tkedr2 = (tip - 2.0 * tk0 + tim) * a.inv_dr2;
    const double ddisdr = (dip - dim) * a.inv_2dr, d2disdr2 = (dip - 2.0 * ds0 + dim) * a.inv_dr2;
    const double dtkedthe = (tjp - tjm) * a.inv_2dthe;
    const double d2tkedthe2 = (tjp - 2.0 * tk0 + tjm) * a.inv_dthe2;
    const double ddisdthe = (djp - djm) * a.inv_2dthe;
    const double d2disdthe2 = (djp - 2.0 * ds0 + djm) * a.inv_dthe2;
    const double dtkedphi = (tkp - tkm) * a.inv_2dphi;
    const double d2tkedphi2 = (tkp - 2.0 * tk0 + tkm) * a.inv_dphi2;
    const double ddisdphi = (dkp - dkm) * a.inv_2dphi;
    const double d2disdphi2 = (dkp - 2.0 * ds0 + dkm) * a.inv_dphi2;

    const double dudr = (uip - uim) * a.inv_2dr;
    const double dvdr = (vip - vim) * a.inv_2dr;
    const double dwdr = (wip - wim) * a.inv_2dr;
    const double dudthe = (ujp - ujm) * a.inv_2dthe;
    const double dvdthe = (vjp - vjm) * a.inv_2dthe;
    const double dwdthe = (wjp - wjm) * a.inv_2dthe;
    const double dudphi = (ukp - ukm) * a.inv_2dphi;
    const double dvdphi = (vkp - vkm) * a.inv_2dphi;
    const double dwdphi = (wkp - wkm) * a.inv_2dphi;
    const double v_invrm = v0 * g.inv_rm;
    const double w_invrs = w0 * g.inv_rmsinthe;
    const double two_inv_rm = 2.0 * g.inv_rm;
    const double transport_tke = u0 * dtkedr + v_invrm * dtkedthe + w_invrs * dtkedphi;
    const double transport_dis = u0 * ddisdr + v_invrm * ddisdthe + w_invrs * ddisdphi;
    const double diffusion_tke = d2tkedr2 + dtkedr * two_inv_rm + d2tkedthe2 * g.inv_rm2 +
                                 dtkedthe * g.costhe_inv_rm2sinthe + d2tkedphi2 * g.inv_rm2sinthe2;
    const double diffusion_dis = d2disdr2 + ddisdr * two_inv_rm + d2disdthe2 * g.inv_rm2 +
                                 ddisdthe * g.costhe_inv_rm2sinthe + d2disdphi2 * g.inv_rm2sinthe2;

    const double C_nue = 0.028, dis_min = 1.0e-10, nue_gas_phys = 1.8e-5;
    const double L_m = a.L_m;
    const double nue_here = isfinite(nv) ? dmax(0.0, nv) : 0.0;
    const double tke_s = dmax(tk0, dis_min);
    const double dis_s = dmax(ds0, dis_min);
    const double dudr_s = dudr, dvdr_s = dvdr, dwdr_s = dwdr;
    const double dudthe_s = dudthe * g.inv_rm, dvdthe_s = dvdthe * g.inv_rm;
    const double dwdthe_s = dwdthe * g.inv_rm;
    const double dudphi_s = dudphi * g.inv_rmsinthe, dvdphi_s = dvdphi * g.inv_rmsinthe;
    const double dwdphi_s = dwdphi * g.inv_rmsinthe;
    const double dtkedthe_s = dtkedthe * g.inv_rm, ddisdthe_s = ddisdthe * g.inv_rm;
    const double dtkedphi_s = dtkedphi * g.inv_rmsinthe, ddisdphi_s = ddisdphi * g.inv_rmsinthe;
    const double grad_dot = dtkedr * ddisdr + dtkedthe_s * ddisdthe_s + dtkedphi_s * ddisdphi_s;
    double cnue = (MODEL == ATJUP_TURB_K_EPSILON) ? C_nue * tke_s * tke_s / dis_s
                                                         : tke_s / dis_s;
    cnue = dmin(cnue, a.nue_max);
    const double der = 0.66667 * (dudr_s + dvdthe_s + dwdphi_s);
    const double P_full = dmax(0.0,
          (cnue * (2.0 * dudr_s - der) - 0.66667 * tk0) * dudr_s
        + (cnue * (dudthe_s + dvdr_s)) * dudthe_s
        + (cnue * (dudphi_s + dwdr_s)) * dudphi_s
        + (cnue * (2.0 * dvdthe_s - der) - 0.66667 * tk0) * dvdthe_s
        + (cnue * (dvdr_s + dudthe_s)) * dvdr_s
        + (cnue * (dvdphi_s + dwdthe_s)) * dvdphi_s
        + (cnue * (2.0 * dwdphi_s - der) - 0.66667 * tk0) * dwdphi_s
        + (cnue * (dwdr_s + dudphi_s)) * dwdr_s
        + (cnue * (dwdthe_s + dvdphi_s)) * dwdthe_s);

    const double y_mount = layer_h(a, topo) * 1.0e3;
    const double dz_layer = dmax(1.0, layer_dz_m(a, i - 1 > 0 ? i - 1 : 0));
    const double y_phys = dmax(layer_h(a, i) * 1.0e3 - y_mount, dz_layer);
    const double y_star = y_phys / L_m;

    double dtre, ddre, tke_src, dis_src, c_w_prod;
    if (MODEL == ATJUP_TURB_K_EPSILON) {               // Chien 1982
        const double sig_k = 1.0, sig_w = 1.3, C_eps_1 = 1.35, C_eps_2 = 1.80;
        dtre = a.inv_re + nue_here / sig_k;
        ddre = a.inv_re + nue_here / sig_w;
        const double d_plus = y_phys * a.vel_star[(size_t)j * a.KP + k] / nue_gas_phys;
        const double Re_T = tke_s * tke_s * a.u_0 * L_m / (dis_s * nue_gas_phys);
        const double f_2 = 1.0 - 0.4 / 1.8 * exp(-Re_T * Re_T / 36.0);
        const double y_star2 = y_star * y_star;
        const double L_k = -2.0 * tk0 / y_star2;
        const double L_w = -2.0 * ds0 / y_star2 * exp(-0.5 * d_plus);
        const double P_w = C_eps_1 * ds0 / tke_s * P_full;
        const double Y_w = C_eps_2 * f_2 * ds0 * ds0 / tke_s;
        tke_src = P_full - ds0 + L_k / a.re_turb;
        dis_src = P_w - Y_w + L_w / a.re_turb;
        c_w_prod = C_eps_1;
    } else if (MODEL == ATJUP_TURB_K_OMEGA) {          // Wilcox
        const double sig_k = 0.6, sig_w = 0.5, bet_star = 0.09, gam = 0.52, bet_0 = 0.0708;
        dtre = a.inv_re + sig_k * nue_here;
        ddre = a.inv_re + sig_w * nue_here;
        const double S11 = dudr_s, S22 = dvdthe_s, S33 = dwdphi_s;
        const double S12 = 0.5 * (dudthe_s + dvdr_s);
        const double S13 = 0.5 * (dudphi_s + dwdr_s);
        const double S23 = 0.5 * (dvdphi_s + dwdthe_s);
        const double S_mag = sqrt(2.0 * (S11 * S11 + S22 * S22 + S33 * S33 +
                                         2.0 * (S12 * S12 + S13 * S13 + S23 * S23)));
        const double W12 = dudthe_s - dvdr_s;
        const double W13 = dudphi_s - dwdr_s;
        const double W23 = dvdphi_s - dwdthe_s;
        const double Omega = sqrt(W12 * W12 + W13 * W13 + W23 * W23);
        const double bd = bet_star * dis_s;
        const double chi_w = fabs(Omega * Omega * S_mag / (bd * bd * bd));   // pow(bd, 3)
        const double f_bet = (1.0 + 85.0 * chi_w) / (1.0 + 100.0 * chi_w);
        const double bet_wc = bet_0 * f_bet;
        const double sig_d = (grad_dot <= 0.0) ? 0.0 : 0.125;
        const double P_k = dmin(P_full, 20.0 * bet_star * tke_s * dis_s);
        const double Y_k = bet_star * tke_s * dis_s;
        const double P_w = gam * dis_s / tke_s * P_k;
        const double Y_w = bet_wc * dis_s * dis_s;
        const double D_w = sig_d / dis_s * grad_dot;
        tke_src = P_k - Y_k;
        dis_src = P_w - Y_w + D_w;
        c_w_prod = gam;
    } else {                                                   // SST, Menter 1994
        const double bet_star = 0.09, sig_k1 = 1.176, sig_k2 = 1.0, sig_w1 = 2.0, sig_w2 = 1.168;
        const double bet1 = 0.0333, bet2 = 0.0368, gam1 = 0.413, gam2 = 0.2;
        const double nue_air_nd = nue_gas_phys / (a.u_0 * L_m);
        const double CD_kw = dmax(2.0 * sig_w2 / dis_s * grad_dot, 1.0e-20);
        const double arg1 = dmin(dmax(sqrt(dmax(tk0, 0.0)) / (bet_star * dis_s * y_star),
                                      500.0 * nue_air_nd / (y_star * y_star * dis_s)),
                                 4.0 * sig_w2 * tke_s / (CD_kw * y_star * y_star));
        const double a2 = arg1 * arg1;
        const double F1 = tanh(a2 * a2);                                     // pow(arg1, 4)
        const double sig_k = F1 * sig_k1 + (1.0 - F1) * sig_k2;
        const double sig_w = F1 * sig_w1 + (1.0 - F1) * sig_w2;
        dtre = a.inv_re + nue_here / sig_k;
        ddre = a.inv_re + nue_here / sig_w;
        const double P_k = dmin(P_full, 20.0 * bet_star * tke_s * dis_s);
        const double Y_k = bet_star * tke_s * dis_s;
        const double P_w = (F1 * gam1 + (1.0 - F1) * gam2) * P_k * dis_s / tke_s;
        const double Y_w = (F1 * bet1 + (1.0 - F1) * bet2) * dis_s * dis_s;
        const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_s * grad_dot;
        tke_src = P_k - Y_k;
        dis_src = P_w - Y_w + D_w;
        c_w_prod = F1 * gam1 + (1.0 - F1) * gam2;
    }
    if (a.turb_buoy) {                                         // RHS_Jup_Turb.cpp:963-981
        const int ip = (i + 1 < a.im - 1) ? i + 1 : a.im - 1, imn = (i - 1 > 0) ? i - 1 : 0;
        const double dz_m = (layer_h(a, ip) - layer_h(a, imn)) * 1.0e3;
        const size_t rs = (size_t)a.jm * a.KP;
        const double T_K = dmax(a.t[x.c] * a.t_ref, 1.0);
        const double dTdz = (a.t[x.c + (ip - i) * rs] - a.t[x.c - (i - imn) * rs]) * a.t_ref /
                            dmax(dz_m, 1.0);
        const double N2 = a.g / T_K * (dTdz + a.g / a.cp_mix);
        const double tscale = L_m / a.u_0;
        const double G_b = -(cnue / a.turb_buoy_prt) * N2 * tscale * tscale;
        if (isfinite(G_b)) {
            tke_src += G_b;
            dis_src += c_w_prod * dis_s / tke_s * dmax(G_b, 0.0);
        }
    }
    const double tke_src_max = 20.0 * tke_s * dis_s;
    const double dis_src_max = 20.0 * dis_s * dis_s;
    if (!isfinite(tke_src)) tke_src = 0.0;
    if (!isfinite(dis_src)) dis_src = 0.0;
    tke_src = dmax(-tke_src_max, dmin(tke_src_max, tke_src));
    dis_src = dmax(-dis_src_max, dmin(dis_src_max, dis_src));
    if (a.stage == 3) {
        a.prod[x.c] = P_full;
        a.tke_source[x.c] = tke_src;
        a.dis_source[x.c] = dis_src;
    }
    rk_update(a, ST, x.c, -transport_tke + diffusion_tke * dtre + tke_src);
    rk_update(a, SD, x.c, -transport_dis + diffusion_dis * ddre + dis_src);
}

}  // namespace

// Field ids of the transported scalars in ATJUP_S_* order, then k*, omega*.
const int kScalarField[ATJUP_S_COUNT + 2] = {
    ATJUP_F_H2O, ATJUP_F_H2O_CLOUD, ATJUP_F_H2O_ICE, ATJUP_F_H2S, ATJUP_F_NH3,
    ATJUP_F_NH3_CLOUD, ATJUP_F_NH3_ICE, ATJUP_F_CH4, ATJUP_F_CH4_CLOUD, ATJUP_F_CH4_ICE,
    ATJUP_F_NH4SH, ATJUP_F_TKE, ATJUP_F_DIS};

namespace {
PhysStage stage_args(AtjupCtx* c, int stage, const double* const* vin) {
    const AtjupParams& P = c->P;
    const AtjupPhysics& H = c->phys;
    PhysStage a{};
    a.u = vin[1];
    a.v = vin[2];
    a.w = vin[3];
    for (int s = 0; s < ATJUP_S_COUNT + 2; s++) {
        const int id = kScalarField[s];
        double* live = c->f[id];
        const double* in[4] = {live, c->S1[s], c->S2[s], c->S1[s]};
        double* out[4] = {c->S1[s], c->S2[s], c->S1[s], live};
        a.q_in[s] = in[stage];
        a.q_out[s] = out[stage];
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

// species_stage_kernel of one RK stage (what = 0) or closure_stage_kernel (what = 1)
int launch_phys_stage(AtjupCtx* c, int stage, const double* const* vin, int what) {
    const AtjupParams& P = c->P;
    const PhysStage a = stage_args(c, stage, vin);
    const dim3 block(128, 2);
    const dim3 grid((P.km + 127) / 128, (P.jm + 1) / 2, P.im);
    if (what == 0) {
        const dim3 sgrid(grid.x, grid.y, P.im * ATJUP_S_COUNT);
        species_stage_kernel<<<sgrid, block, 0, c->stream>>>(a);
        c->launches++;
        ATJUP_CHECK_LAUNCH("species_stage_kernel");
    } else {
        switch (a.turb_model) {
        case ATJUP_TURB_K_EPSILON:
            closure_stage_kernel<ATJUP_TURB_K_EPSILON><<<grid, block, 0, c->stream>>>(a);
            break;
        case ATJUP_TURB_K_OMEGA:
            closure_stage_kernel<ATJUP_TURB_K_OMEGA><<<grid, block, 0, c->stream>>>(a);
            break;
        default:
            closure_stage_kernel<ATJUP_TURB_K_OMEGA_SST><<<grid, block, 0, c->stream>>>(a);
        }
        c->launches++;
        ATJUP_CHECK_LAUNCH("closure_stage_kernel");
    }
    return ATJUP_OK;
}

}  // namespace atjup
