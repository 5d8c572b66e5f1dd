// The loop's microphysics on the device: radiation, precipitation, the NH4SH equilibrium, the
// chemistry mass fluxes and the species clamp.
//
//   radiation_kernel      Radiation<cJupiterModel>::run (Radiation.h:251-456)
//   precip_kernel         Precipitation<cJupiterModel>::run / column (Precipitation.h:191-445)
//   nh4sh_kernel          ChemistryJup::EquilibriumNH4SH("loop") (ChemistryJup.h:291-373)
//   difflux_kernel        the diffusive fluxes of DiffMassFluxJup (ChemistryJup.h:375-538, 756-780)
//   massflux_kernel       ChemMassRateJup: reaction rate + diffusive flux (ChemistryJup.h:59-281)
//   fluxlim_kernel        FluxLimiter<cJupiterModel>::nh4sh (FluxLimiter.h)
//   clamp_species_kernel  clampNegativeSpecies (FileIO_Jup.cpp:494-548)
//   diagnostics_kernel    cJupiterModel::Forces (InitValues_Jup.cpp:742-812) and Latent_Heat
//                         (Thermo_Jup.cpp:89-232): output fields only
//
// Radiation and precipitation are vertical sweeps through a column (the thermal fluxes down then
// up, the falling hydrometeor fluxes top-down), so each is one thread per (j, k) column, k fastest
// so that a warp's loads at one level are consecutive, with the column's levels in local arrays
// and the fluxes carried in registers. The rest are pointwise or 7-point stencils, one thread per
// cell. The column's sweep order and every expression's operand order follow the reference, and
// the file is compiled without FMA contraction: the precipitation's fluxes cancel to exactly zero
// when a layer evaporates all the rain that reaches it, and the next layer branches on that zero.
#include "ctx.cuh"
#include "dd_exp10.cuh"

namespace atjup {
namespace {

constexpr int MAX_IM = 64;   // levels a column kernel holds (the reference grid has 41)

__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }

struct MicroArgs {
    const double *p_stat, *rho_mix, *u, *v, *w;
    double* t;
    double* q[ATJUP_S_COUNT];          // species (ATJUP_S_* order)
    double* sprec[9];
    double *Q_rad, *Q_precip;
    double *difflux[3], *massflux[3], *fluxlim;
    const int32_t* topo;
    const float* layer_h;
    const uint8_t* solid;
    const double* rad;
    const double* sin_the;             // [jm] sin(the_j)
    const double* cos_lat;             // [jm] max(0, sin(pi j / (jm - 1))): the solar geometry
    const GeoIJ* geo;
    AtjupMicro mc;
    int im, jm, km, KP, local_rho;
    double t_ref, g, r_mix, cp_mix, L_atm, u_0, dr, dthe, dphi;
};

__device__ __forceinline__ double layer_dz_m(const MicroArgs& a, int i) {
    if (i < 0 || i > a.im - 2) return -1.0;
    return (double)(a.layer_h[i + 1] - a.layer_h[i]) * 1.0e3;
}

// ATPhys::saturation_vapour_pressure (ATPhys.h:49-52) [bar]
__device__ __forceinline__ double svp(double T, double C, double L0, double R, double da, double db) {
    return exp(C + (-L0 / T + da * log(T) + db * T) / (1e-3 * R));
}

__global__ void radiation_kernel(MicroArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (k >= a.km) return;
    const double sigma = 5.670374419e-8, P0_phys = 1.0e5, he_ratio = 0.6, C_cia = 3.5e-6;
    const double kappa_ch4 = 0.003, kappa_nh3 = 1.5, kappa_cloud = 25.0, kappa_ice = 12.0;
    const double tau_cloud_cap = 0.4, opac_cal = 0.025, pi_ = 3.14159265358979323846;
    const AtjupMicro& mc = a.mc;
    const double comp = mc.x_H2 * mc.x_H2 + he_ratio * mc.x_H2 * mc.x_He;
    const double cia_coeff = C_cia * mc.cia_strength * comp / a.g;
    const double opac_mult = mc.opacity_strength;
    const size_t plane = (size_t)a.jm * a.KP, c0 = (size_t)j * a.KP + k;
    int i_base = a.topo[(size_t)j * a.km + k];
    if (i_base < 0) i_base = 0;
    const int i_top = a.im - 1;
    if (i_base >= i_top) return;
    double B[MAX_IM], eps[MAX_IM], Fd[MAX_IM + 1], Fu[MAX_IM + 1], Fsw[MAX_IM + 2];
    // the levels are independent here: unrolled, the loads of four levels are in flight together
#pragma unroll 4
    for (int i = i_base; i <= i_top; i++) {
        const size_t c = c0 + (size_t)i * plane;
        const double T = a.t[c] * a.t_ref;
        B[i] = sigma * T * T * T * T;
        const double P_lo = a.p_stat[c] * P0_phys;
        const double P_hi = (i < i_top) ? a.p_stat[c + plane] * P0_phys : 0.0;
        double dP = P_lo - P_hi;
        if (dP < 0.0) dP = 0.0;
        const double P_mean = 0.5 * (P_lo + P_hi);
        const double dm = dP / a.g;
        const double tau_cia = (T > 0.0) ? cia_coeff * (P_mean / T) * dP : 0.0;
        const double rho_c = a.rho_mix[c];
        const double inv_rho = (rho_c > 0.0 && isfinite(rho_c)) ? 1.0 / rho_c : 0.0;
        const double q_ch4 = dmax(0.0, a.q[ATJUP_S_CH4][c]) * inv_rho;
        const double q_nh3 = dmax(0.0, a.q[ATJUP_S_NH3][c]) * inv_rho;
        const double tau_gas = opac_mult * opac_cal * (kappa_ch4 * q_ch4 + kappa_nh3 * q_nh3) * dm;
        const double q_liq = (dmax(0.0, a.q[ATJUP_S_H2O_CLOUD][c]) + dmax(0.0, a.q[ATJUP_S_NH3_CLOUD][c]) +
                              dmax(0.0, a.q[ATJUP_S_CH4_CLOUD][c])) * inv_rho;
        const double q_ice = (dmax(0.0, a.q[ATJUP_S_H2O_ICE][c]) + dmax(0.0, a.q[ATJUP_S_NH3_ICE][c]) +
                              dmax(0.0, a.q[ATJUP_S_CH4_ICE][c])) * inv_rho;
        double tau_cloud = opac_mult * opac_cal * (kappa_cloud * q_liq + kappa_ice * q_ice) * dm;
        if (tau_cloud > tau_cloud_cap) tau_cloud = tau_cloud_cap;
        eps[i] = 1.0 - exp(-(tau_cia + tau_gas + tau_cloud));
    }
    for (int i = i_base; i <= i_top + 1; i++) Fsw[i] = 0.0;
    if (mc.solar_on != 0) {
        const double F_sun_toa = mc.solar_strength * mc.S_solar * (1.0 - mc.albedo_bond) * a.cos_lat[j] / pi_;
        for (int i = i_base; i <= i_top + 1; i++) {
            const double p_bar = (i <= i_top) ? a.p_stat[c0 + (size_t)i * plane] : 0.0;
            Fsw[i] = F_sun_toa * exp(-mc.sw_tau_per_bar * dmax(0.0, p_bar));
        }
    }
    Fd[i_top + 1] = 0.0;
    for (int i = i_top; i >= i_base; i--) Fd[i] = Fd[i + 1] * (1.0 - eps[i]) + eps[i] * B[i];
    if (mc.rad_bottom == 1) Fu[i_base] = dmax(0.0, 2.0 * B[i_base] - Fd[i_base + 1]);
    else Fu[i_base] = Fd[i_base] + mc.F_int + Fsw[i_base];
    for (int i = i_base; i <= i_top; i++) Fu[i + 1] = Fu[i] * (1.0 - eps[i]) + eps[i] * B[i];
    for (int i = i_base; i <= i_top; i++) {
        const double net_bot = Fu[i] - Fd[i];
        const double net_top = Fu[i + 1] - Fd[i + 1];
        double dz = (i < i_top) ? layer_dz_m(a, i) : layer_dz_m(a, i - 1);
        if (dz <= 0.0) dz = 1.0;
        const double Q_sw = (Fsw[i + 1] - Fsw[i]) / dz;
        a.Q_rad[c0 + (size_t)i * plane] = (net_bot - net_top) / dz + Q_sw;
    }
    for (int i = 0; i < i_base; i++) a.Q_rad[c0 + (size_t)i * plane] = 0.0;
}

// The inputs of one level of a column sweep, loaded ahead of the level's computation.
struct PrecipLevel {
    double t, p, vap, cld, ice, rho;
};

__device__ __forceinline__ PrecipLevel precip_load(const MicroArgs& a, const double* vap,
                                                   const double* cld, const double* ice, size_t c) {
    PrecipLevel L;
    L.t = a.t[c];
    L.p = a.p_stat[c];
    L.vap = vap[c];
    L.cld = cld[c];
    L.ice = ice[c];
    L.rho = a.local_rho ? a.rho_mix[c] : 0.0;
    return L;
}

// The three gases' sweeps of a column are independent except for Q_precip, the sum of their
// latent heating. So a block is PR_COLS columns x 3 gases (threadIdx.y = gas: H2O, NH3, CH4), the
// three threads of a column walk its levels in step, and at each level the H2O thread adds the
// three contributions in the reference's order ((0 + H2O) + NH3) + CH4 from shared memory
// (double-buffered by level parity, one barrier per level). Within a sweep the inputs of a level
// depend only on the state before the sweep: each level's loads are issued two levels ahead of
// its computation (and so ahead, in program order, of the stores of the level in between, which
// touch other cells), so a column waits for one memory round trip per sweep, not one per level.
constexpr int PRECIP_AHEAD = 2;
constexpr int PR_COLS = 64;

__global__ void __launch_bounds__(PR_COLS * 3, 4) precip_kernel(MicroArgs a) {
    __shared__ double contrib[2][3][PR_COLS];
    const int tx = threadIdx.x, gq = threadIdx.y;
    const int k = blockIdx.x * PR_COLS + tx, j = blockIdx.y;
    const bool col = k < a.km;
    const size_t plane = (size_t)a.jm * a.KP, c0 = (size_t)j * a.KP + (col ? k : 0);
    const AtjupGasParams& gs = a.mc.gas[gq];
    const int sv = gq == 0 ? ATJUP_S_H2O : (gq == 1 ? ATJUP_S_NH3 : ATJUP_S_CH4);
    double *vap = a.q[sv], *cld = a.q[sv + 1], *ice = a.q[sv + 2];
    double *Sv = a.sprec[3 * gq], *Sc = a.sprec[3 * gq + 1], *Si = a.sprec[3 * gq + 2];
    if (col) {
        for (int i = 0; i < a.im; i++) {
            const size_t c = c0 + (size_t)i * plane;
            if (gq == 0) a.Q_precip[c] = 0.0;
            Sv[c] = 0.0;
            Sc[c] = 0.0;
            Si[c] = 0.0;
        }
    }
    int i_base = col ? a.topo[(size_t)j * a.km + k] : a.im;
    if (i_base < 0) i_base = 0;
    const int i_top = a.im - 1;
    const bool live = col && i_base < i_top;   // the column has levels to sweep
    const AtjupMicro& mc = a.mc;
    const double P_max_flux = 1.0e-4, dep_frac = 1.0, ratio_cap = 5.0, rs = mc.precip_rate_scale;
    const double c_c_au = 2.0e-8, c_i_au = 5.0e-8, q_c_crit = 5.0e-4, c_ac = 1.0e-7;
    const double c_rim = 1.0e-8, z_csg = 2.5e-8, a_ev = 2.76e-3, c_melt_K = 0.2, c_frz_K = 0.2;
    const double P_ref = 1.0e-4, v_fall = 2.0;
    const double nd = (a.L_atm * 1.0e3) / a.u_0;
    const double Lf = gs.ls - gs.lv;
    double Pr = 0.0, Ps = 0.0, Pg = 0.0;
    // ring of the next PRECIP_AHEAD levels' inputs (level i - q in slot q - 1)
    PrecipLevel ahead[PRECIP_AHEAD];
#pragma unroll
    for (int q = 0; q < PRECIP_AHEAD; q++) {
        const int il = i_top - 1 - q;
        if (live && il >= i_base) ahead[q] = precip_load(a, vap, cld, ice, c0 + (size_t)il * plane);
    }
    // every thread of the block walks the same levels (the barrier below is block-wide); a
    // column takes part from its top level down to its base
    for (int i = i_top - 1; i >= 0; i--) {
        const bool act = live && i >= i_base;
        const size_t c = c0 + (size_t)i * plane;
        PrecipLevel L{};
        if (act) {
            L = ahead[0];
#pragma unroll
            for (int q = 0; q < PRECIP_AHEAD - 1; q++) ahead[q] = ahead[q + 1];
            if (i - PRECIP_AHEAD >= i_base)
                ahead[PRECIP_AHEAD - 1] = precip_load(a, vap, cld, ice, c - (size_t)PRECIP_AHEAD * plane);
        }
        const double dz = dmax(0.0, layer_dz_m(a, i));
        if (dz <= 0.0) continue;          // the same for every thread: no barrier is skipped unevenly
        double q_heat = 0.0;
        if (act) {
            const double T = L.t * a.t_ref;
            const double p_u = L.p;
            const double q_v = dmax(0.0, L.vap), q_c = dmax(0.0, L.cld), q_i = dmax(0.0, L.ice);
            const double E_r = svp(T, gs.C, gs.L0, gs.R, gs.del_alf, gs.del_bet);
            double rho = a.r_mix;
            if (a.local_rho) {
                const double r = L.rho;
                if (r > 0.0 && isfinite(r)) rho = r;
            }
            const double q_sat = (p_u > E_r) ? rho * gs.ep * E_r / p_u : q_v;
            const double F_r_in = Pr, F_s_in = Ps, F_g_in = Pg;
            const double Rain = dmin(ratio_cap, F_r_in / P_ref);
            const double Snow = dmin(ratio_cap, F_s_in / P_ref);
            const double Graupel = dmin(ratio_cap, F_g_in / P_ref);
            const double Rain_79 = (Rain > 0.0) ? pow(Rain, 7.0 / 9.0) : 0.0;
            const double Rain_49 = (Rain > 0.0) ? pow(Rain, 4.0 / 9.0) : 0.0;
            const bool warm = (T >= gs.t_0);
            const double S_c_au = (warm && q_c > q_c_crit) ? (rs * c_c_au) * (q_c - q_c_crit) : 0.0;
            const double S_i_au = (!warm && T >= gs.t_00) ? (rs * c_i_au) * q_i : 0.0;
            const double S_ac = warm ? (rs * c_ac) * q_c * Rain_79 : 0.0;
            const double S_s_rim = !warm ? (rs * c_rim) * q_c * Snow : 0.0;
            const double S_g_rim = !warm ? (rs * c_rim) * q_c * Graupel : 0.0;
            const double S_csg = (!warm && q_c > q_c_crit) ? (rs * z_csg) * q_c * Snow : 0.0;
            const double f_melt = warm ? dmin(1.0, c_melt_K * (T - gs.t_0)) : 0.0;
            const double f_frz = warm ? 0.0 : dmin(1.0, c_frz_K * (gs.t_0 - T));
            const double F_s_melt = f_melt * F_s_in, F_g_melt = f_melt * F_g_in;
            const double F_r_frz = f_frz * F_r_in;
            const double F_r_avail = dmax(0.0, F_r_in - F_r_frz + F_s_melt + F_g_melt + (S_c_au + S_ac) * dz);
            const double S_ev_raw = (warm && Rain > 0.0 && q_v < q_sat) ? a_ev * (q_sat - q_v) * Rain_49 : 0.0;
            const double F_ev_sat = dmax(0.0, q_sat - q_v) * v_fall;
            const double F_ev = dmin(dmin(S_ev_raw * dz, F_r_avail), F_ev_sat);
            const double S_ev = F_ev / dz;
            q_heat = Lf * (S_s_rim + S_g_rim + S_csg) + Lf * (F_r_frz - F_s_melt - F_g_melt) / dz -
                     gs.lv * F_ev / dz;
            const double tau = dz / v_fall;
            const double d_c = dmin(dep_frac * q_c, (S_c_au + S_ac + S_s_rim + S_g_rim + S_csg) * tau);
            const double d_i = dmin(dep_frac * q_i, S_i_au * tau);
            if (mc.precip_coupling_on) {
                Sc[c] = -dmax(0.0, d_c) / tau * nd;
                Si[c] = -dmax(0.0, d_i) / tau * nd;
                Sv[c] = +S_ev * nd;
            } else {
                cld[c] = q_c - dmax(0.0, d_c);
                ice[c] = q_i - dmax(0.0, d_i);
                vap[c] = q_v + S_ev * tau;
            }
            const double F_r = F_r_in - F_r_frz + F_s_melt + F_g_melt - F_ev + (S_c_au + S_ac) * dz;
            const double F_s = F_s_in - F_s_melt + (S_i_au + S_s_rim - S_csg) * dz;
            const double F_g = F_g_in - F_g_melt + F_r_frz + (S_g_rim + S_csg) * dz;
            Pr = dmin(P_max_flux, dmax(0.0, F_r));
            Ps = dmin(P_max_flux, dmax(0.0, F_s));
            Pg = dmin(P_max_flux, dmax(0.0, F_g));
        }
        const int b = i & 1;
        contrib[b][gq][tx] = q_heat;
        __syncthreads();
        if (act && gq == 0)   // Q_precip += H2O, then NH3, then CH4 (Q_precip was zeroed above)
            a.Q_precip[c] = ((0.0 + contrib[b][0][tx]) + contrib[b][1][tx]) + contrib[b][2][tx];
    }
}

// one thread per cell over the padded block; k < km
__device__ __forceinline__ bool cell_index(const MicroArgs& a, int& i, int& j, int& k, size_t& c) {
    k = blockIdx.x * blockDim.x + threadIdx.x;
    j = blockIdx.y;
    i = blockIdx.z;
    if (k >= a.km) return false;
    c = ((size_t)i * a.jm + j) * a.KP + k;
    return true;
}

// The sign of f(x) of ChemistryJup.h:297-300, the only use the bisection makes of it. K_p =
// 10^(14.82 - 4705 / T); the reference takes it from the C library's pow, which rounds (nearly
// always) correctly. CUDA's exp10 is within 1 ulp of 10^y, so B = K_p atm^2 formed from it is
// within about 4 ulp (1e-15 relative) of B formed from the correctly rounded K_p; when
// |A - B| exceeds 1e-14 B, the sign of A - B is therefore the correctly rounded one. Only
// within that margin of the root is K_p recomputed through the correctly rounded
// double-double exponential (dd_exp10.cuh). Non-finite values fail the margin test and take
// the double-double path too.
__device__ __forceinline__ double nh4sh_f(double x, double a_, double b_, double T0, double heat) {
    const double R_univ = 8314.46, atm = 101325.0;
    const double T = T0 + heat * x, RT = R_univ * T;
    const double A = (a_ - x) * (b_ - x) * RT * RT;
    const double y = 14.82 - 4705.0 / T;
    const double B_fast = exp10(y) * atm * atm;
    if (fabs(A - B_fast) > 1.0e-14 * B_fast) return A - B_fast;
    return A - ddx::exp10(y) * atm * atm;
}

__global__ void nh4sh_kernel(MicroArgs a, double L_f) {
    int i, j, k;
    size_t c;
    if (!cell_index(a, i, j, k, c) || a.solid[c]) return;
    const AtjupMicro& mc = a.mc;
    double *nh3 = a.q[ATJUP_S_NH3], *h2s = a.q[ATJUP_S_H2S], *nh4sh = a.q[ATJUP_S_NH4SH];
    const double T0 = a.t[c] * a.t_ref;
    if (!(T0 > 0.0)) return;
    double rho = a.rho_mix[c];
    if (!(rho > 0.0) || !isfinite(rho)) rho = a.r_mix;
    const double av = dmax(0.0, nh3[c]) / mc.m_nh3;
    const double bv = dmax(0.0, h2s[c]) / mc.m_h2s;
    const double sv = dmax(0.0, nh4sh[c]) / mc.m_nh4sh;
    const double heat = L_f * mc.m_nh4sh / (a.cp_mix * rho);
    const double f0 = nh4sh_f(0.0, av, bv, T0, heat);
    double lo, hi;
    if (f0 > 0.0) {
        lo = 0.0;
        hi = dmin(av, bv);
    } else if (sv > 0.0) {
        if (nh4sh_f(-sv, av, bv, T0, heat) <= 0.0) { lo = hi = -sv; }
        else { lo = -sv; hi = 0.0; }
    } else {
        return;
    }
    if (hi > lo)
        for (int it = 0; it < 80; it++) {
            const double xm = 0.5 * (lo + hi);
            if (nh4sh_f(xm, av, bv, T0, heat) > 0.0) lo = xm; else hi = xm;
            if (hi - lo <= 1.0e-15 * dmax(av, dmax(bv, sv))) break;
        }
    const double x = (f0 > 0.0) ? lo : hi;
    if (x == 0.0) return;
    nh3[c] = dmax(0.0, nh3[c] - mc.m_nh3 * x);
    h2s[c] = dmax(0.0, h2s[c] - mc.m_h2s * x);
    nh4sh[c] = dmax(0.0, nh4sh[c] + mc.m_nh4sh * x);
    a.t[c] = (T0 + heat * x) / a.t_ref;
}

__global__ void difflux_kernel(MicroArgs a) {
    int i, j, k;
    size_t c;
    if (!cell_index(a, i, j, k, c)) return;
    if (k > a.km - 2 || j < 1 || j > a.jm - 2 || i < 1 || i > a.im - 2) return;
    if (!(a.t[c] > 0.0) || a.solid[c]) {
        for (int q = 0; q < 3; q++) a.difflux[q][c] = 0.0;
        return;
    }
    const double rm = a.rad[i];
    const double sinthe = a.sin_the[j];
    const double costhe = a.geo[(size_t)i * a.jm + j].costhe;
    const double rmsinthe = rm * dmax(sinthe, a.mc.polar_divisor_floor);
    const size_t plane = (size_t)a.jm * a.KP, row = c - k;
    const int ke = (k >= a.km - 2) ? 0 : k + 1, kw = (k == 0) ? a.km - 2 : k - 1;
    const double D[3] = {a.mc.D_h2s, a.mc.D_nh3, a.mc.D_nh4sh};
    const int sp[3] = {ATJUP_S_H2S, ATJUP_S_NH3, ATJUP_S_NH4SH};
    for (int q = 0; q < 3; q++) {
        const double* s = a.q[sp[q]];
        const double c0 = s[c];
        const double d2cdr2 = (s[c + plane] - 2.0 * c0 + s[c - plane]) / (a.dr * a.dr) * 1.0;
        const double d2cdthe2 = (s[c + a.KP] - 2.0 * c0 + s[c - a.KP]) / (a.dthe * a.dthe);
        const double d2cdphi2 = (s[row + ke] - 2.0 * c0 + s[row + kw]) / (a.dphi * a.dphi);
        const double dcdr = (s[c + plane] - s[c - plane]) / (2.0 * a.dr) * 1.0;
        const double dcdthe = (s[c + a.KP] - s[c - a.KP]) / (2.0 * a.dthe);
        const double lap = d2cdr2 + 2.0 / rm * dcdr + d2cdthe2 / (rm * rm) +
                           costhe / (rm * rmsinthe) * dcdthe + d2cdphi2 / (rmsinthe * rmsinthe);
        a.difflux[q][c] = D[q] * lap;
    }
}

__global__ void massflux_kernel(MicroArgs a) {
    int i, j, k;
    size_t c;
    if (!cell_index(a, i, j, k, c)) return;
    if (j < 3 || j >= a.jm - 3) {
        for (int q = 0; q < 3; q++) a.massflux[q][c] = 0.0;
        return;
    }
    if (k > a.km - 2 || i < 1 || i > a.im - 2) return;
    const size_t plane = (size_t)a.jm * a.KP, row = c - k;
    const int ke = (k >= a.km - 2) ? 0 : k + 1, kw = (k == 0) ? a.km - 2 : k - 1;
    const uint8_t* S = a.solid;
    if (S[c] && S[c - plane] && S[c + plane] && S[c - a.KP] && S[c + a.KP] && S[row + kw] && S[row + ke]) {
        for (int q = 0; q < 3; q++) a.massflux[q][c] = 0.0;
        return;
    }
    // the reaction rates in kg/(m3 s), ordered like massflux (H2S, NH3, NH4SH); 0 with the
    // equilibrium on and outside the 200..230 K formation window (the gate-zero default)
    double w[3] = {0.0, 0.0, 0.0};
    if (!a.mc.nh4sh_eq) {
        const AtjupMicro& m = a.mc;
        const double t_u = a.t[c] * a.t_ref;
        if (t_u <= m.t_0_nh4sh && t_u >= m.t_00_nh4sh) {
            const double keq = m.m_nh4sh / (m.m_nh3 * m.m_h2s);
            const double kf = 15000.0 * pow(t_u, -0.5) * exp(-3020.0 / t_u);
            const double kb = kf / keq;
            const double nh3 = a.q[ATJUP_S_NH3][c], h2s = a.q[ATJUP_S_H2S][c], nh4sh = a.q[ATJUP_S_NH4SH][c];
            // the concentrations normalised to carry r_mix together (the molar-concentration
            // form is the non-default alternative)
            const double sum_c = nh3 / m.m_nh3 + h2s / m.m_h2s + nh4sh / m.m_nh4sh;
            const double denom = (sum_c == 0.0) ? 0.0 : a.r_mix / sum_c;
            const double c_nh3 = nh3 / m.m_nh3 * denom;
            const double c_h2s = h2s / m.m_h2s * denom;
            const double c_nh4sh = nh4sh / m.m_nh4sh * denom;
            const double R_diff = kf * c_nh3 * c_h2s - kb * c_nh4sh;
            w[0] = -m.m_h2s * R_diff;
            w[1] = -m.m_nh3 * R_diff;
            w[2] = m.m_nh4sh * R_diff;
        }
    }
    for (int q = 0; q < 3; q++) a.massflux[q][c] = w[q] + a.difflux[q][c];
}

__device__ __forceinline__ double superbee_phi(double r) {
    return dmax(0.0, dmax(dmin(2.0 * r, 1.0), dmin(r, 2.0)));
}

__global__ void fluxlim_kernel(MicroArgs a) {
    int i, j, k;
    size_t c;
    if (!cell_index(a, i, j, k, c)) return;
    if (k > a.km - 2 || j < 1 || j > a.jm - 2 || i < 1 || i > a.im - 2) return;
    const double* Q = a.q[ATJUP_S_NH4SH];
    const size_t plane = (size_t)a.jm * a.KP, row = c - k;
    const int n = a.km - 1;
    auto wrap = [&](int kk) { return kk < 0 ? kk + n : (kk >= n ? kk - n : kk); };
    const double eps = 1.0e-12;
    const double q = Q[c];
    const double q_rp = Q[c + plane], q_rm = Q[c - plane], q_tp = Q[c + a.KP], q_tm = Q[c - a.KP];
    const double q_pp = Q[row + wrap(k + 1)], q_pm = Q[row + wrap(k - 1)];
    const double u = a.u[c], v = a.v[c], w = a.w[c];
    const double rm = a.rad[i];
    const double sinthe = dmax(a.mc.polar_divisor_floor, fabs(a.sin_the[j]));
    const double inv_rm = 1.0 / rm;
    const double inv_rmsinthe = 1.0 / (rm * sinthe);
    double corr = 0.0;
    {
        const double df = q_rp - q, db = q - q_rm;
        const double denom = df + (df >= 0.0 ? eps : -eps);
        const double r = (u >= 0.0) ? db / denom : ((i + 2 < a.im ? Q[c + 2 * plane] : q_rp) - q_rp) / denom;
        corr += (1.0 - superbee_phi(r)) * fabs(u) * (df - db) / (2.0 * a.dr);
    }
    {
        const double df = q_tp - q, db = q - q_tm;
        const double denom = df + (df >= 0.0 ? eps : -eps);
        const double q_far = (j + 2 < a.jm) ? Q[c + 2 * a.KP] : ((4.0 / 3.0) * q_tp - (1.0 / 3.0) * q);
        const double r = (v >= 0.0) ? db / denom : (q_far - q_tp) / denom;
        corr += (1.0 - superbee_phi(r)) * fabs(v) * inv_rm * (df - db) / (2.0 * a.dthe);
    }
    {
        const double df = q_pp - q, db = q - q_pm;
        const double denom = df + (df >= 0.0 ? eps : -eps);
        const double r = (w >= 0.0) ? db / denom : (Q[row + wrap(k + 2)] - q_pp) / denom;
        corr += (1.0 - superbee_phi(r)) * fabs(w) * inv_rmsinthe * (df - db) / (2.0 * a.dphi);
    }
    a.fluxlim[c] = corr;
}

__global__ void clamp_species_kernel(MicroArgs a) {
    int i, j, k;
    size_t c;
    if (!cell_index(a, i, j, k, c)) return;
    for (int s = 0; s < ATJUP_S_COUNT; s++)
        if (!(a.q[s][c] >= 0.0)) a.q[s][c] = 0.0;
}

// The output diagnostics: the force densities of Forces and the latent and sensible heating of
// Latent_Heat. One thread per cell; both routines fill i 1..im-2, j 1..jm-2 and the phi ring
// k 0..km-2, Latent_Heat also zeroes its fields at i = 0; other cells keep their values. The
// sine and cosine of the colatitude are the host's (the reference's sin and cos of the.z), and
// every expression keeps the reference's operand order (this file has no FMA contraction), so
// only CUDA's exp differs in its last bit; it feeds the saturation tests of Latent_Heat.
struct DiagArgs {
    const double *t, *u, *v, *w, *p_dyn, *p_stat, *h2o, *nh3;
    const uint8_t* solid;
    const double *rad, *sin_the;
    const GeoIJ* geo;
    double *cor, *cen, *buo, *pgf, *ql, *qs;
    double cc[8];
    double ep_w, lv_w, ls_w, ep_a, lv_a, ls_a, fix_lat, fix_sen;
    double omega, Coriolis, centrifugal, buoyancy, r_mix, R_mix, g, t_ref, p_dyn_to_bar, L_atm;
    double u_0, cp_mix, dr, dthe, dphi;
    int im, jm, km, KP, costhe_abs;
};

__global__ void diagnostics_kernel(DiagArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    if (k >= a.km) return;
    const size_t plane = (size_t)a.jm * a.KP, row = ((size_t)i * a.jm + j) * a.KP, c = row + k;
    if (i == 0) {
        a.ql[c] = 0.0;
        a.qs[c] = 0.0;
        return;
    }
    if (i > a.im - 2 || j < 1 || j > a.jm - 2 || k > a.km - 2) return;
    const int ke = (k >= a.km - 2) ? 0 : k + 1, kw = (k == 0) ? a.km - 2 : k - 1;
    const size_t cp = c + plane, cm = c - plane, cjp = c + a.KP, cjm = c - a.KP;
    const size_t ckp = row + ke, ckm = row + kw;
    const double rm = a.rad[i];
    const double sinthe = a.sin_the[j];
    double costhe = a.geo[(size_t)i * a.jm + j].costhe;
    if (a.costhe_abs && j > 90) costhe = -costhe;
    const double rmsinthe = rm * sinthe;
    // Forces
    const double omega = a.omega;
    const double Cor_r = -2.0 * omega * sinthe * a.w[c];
    const double Cor_the = +2.0 * omega * costhe * a.w[c];
    const double Cor_phi = +2.0 * omega * (-costhe * a.v[c] + sinthe * a.u[c]);
    const double dpdr = (a.p_dyn[cp] - a.p_dyn[cm]) / (2.0 * a.dr);
    const double dpdthe = (a.p_dyn[cjp] - a.p_dyn[cjm]) / (2.0 * a.dthe);
    const double dpdphi = (a.p_dyn[ckp] - a.p_dyn[ckm]) / (2.0 * a.dphi);
    a.cor[c] = a.Coriolis * a.r_mix * sqrt((Cor_r * Cor_r + Cor_the * Cor_the + Cor_phi * Cor_phi) / 3.0);
    a.cen[c] = a.centrifugal * a.r_mix * omega * omega * rm * (1.0 + fabs(sinthe));
    const double tc = a.t[c];
    a.buo[c] = (tc > 0.0) ? a.buoyancy * a.r_mix * a.g * (a.p_stat[c] + a.p_dyn[c] * a.p_dyn_to_bar) /
                                (a.r_mix * a.R_mix * tc * a.t_ref) * 1e5
                          : 0.0;
    const double gth = dpdthe / rm, gph = dpdphi / rmsinthe;
    a.pgf[c] = -sqrt((dpdr * dpdr + gth * gth + gph * gph) / 3.0) * a.p_dyn_to_bar * 1.0e5 /
               (a.L_atm * 1.0e3);
    // Latent_Heat
    const double t_u = tc * a.t_ref;
    const double p_u = a.p_stat[c];
    const double E_Rain = exp(a.cc[0] / t_u + a.cc[1]);
    const double E_Ice = exp(a.cc[2] / t_u + a.cc[3]);
    const double q_Rain = a.ep_w * E_Rain / dmax(p_u - E_Rain, 1.0e-12);
    const double q_Ice = a.ep_w * E_Ice / dmax(p_u - E_Ice, 1.0e-12);
    const double E_Rain_nh3 = exp(a.cc[4] / t_u + a.cc[5]);
    const double E_Ice_nh3 = exp(a.cc[6] / t_u + a.cc[7]);
    const double q_Rain_nh3 = a.ep_a * E_Rain_nh3 / dmax(p_u - E_Rain_nh3, 1.0e-12);
    const double q_Ice_nh3 = a.ep_a * E_Ice_nh3 / dmax(p_u - E_Ice_nh3, 1.0e-12);
    const double u_av = 0.5 * (a.u[cp] + a.u[cm]);
    const double v_av = 0.5 * (a.v[cp] + a.v[cm]);
    const double w_av = 0.5 * (a.w[cp] + a.w[cm]);
    const double velocity_av = -sqrt((u_av * u_av + v_av * v_av + w_av * w_av) / 3.0);
    const double dtdr = (a.t[cp] - a.t[cm]) / (2.0 * a.dr) * 1.0;
    const double dtdthe = (a.t[cjp] - a.t[cjm]) / (2.0 * rm * a.dthe);
    const double dtdphi = (a.t[ckp] - a.t[ckm]) / (2.0 * rmsinthe * a.dphi);
    const double dh2odr = (a.h2o[cp] - a.h2o[cm]) / (2.0 * a.dr) * 1.0;
    const double dh2odthe = (a.h2o[cjp] - a.h2o[cjm]) / (2.0 * rm * a.dthe);
    const double dh2odphi = (a.h2o[ckp] - a.h2o[ckm]) / (2.0 * rmsinthe * a.dphi);
    const double dnh3dr = (a.nh3[cp] - a.nh3[cm]) / (2.0 * a.dr) * 1.0;
    const double dnh3dthe = (a.nh3[cjp] - a.nh3[cjm]) / (2.0 * rm * a.dthe);
    const double dnh3dphi = (a.nh3[ckp] - a.nh3[ckm]) / (2.0 * rmsinthe * a.dphi);
    const double dtemp = dtdr + dtdthe + dtdphi;
    const double dh2o = dh2odr + dh2odthe + dh2odphi;
    const double dnh3 = dnh3dr + dnh3dthe + dnh3dphi;
    const double Lr = a.L_atm * (a.im - 1);
    const double h = a.h2o[c], nn = a.nh3[c];
    double ql = (h >= q_Rain) ? a.lv_w * velocity_av * dh2o * a.u_0 / Lr * a.fix_lat : 0.0;
    double ice = (h >= q_Ice) ? a.ls_w * velocity_av * dh2o * a.u_0 / Lr * a.fix_lat : 0.0;
    if (nn >= q_Rain_nh3) ql = ql + a.lv_a * velocity_av * dnh3 * a.u_0 / Lr * a.fix_lat;
    if (nn >= q_Ice_nh3) ice = ice + a.ls_a * velocity_av * dnh3 * a.u_0 / Lr * a.fix_lat;
    ql = ql + ice;
    double qs = a.r_mix * a.cp_mix * velocity_av * a.u_0 * dtemp * a.t_ref / (Lr * Lr) * a.fix_sen;
    if (a.solid[c] == 1) { ql = 0.0; qs = 0.0; }
    a.ql[c] = ql;
    a.qs[c] = qs;
}

DiagArgs diag_args(AtjupCtx* c) {
    const AtjupParams& P = c->P;
    const AtjupMicro& mc = c->micro;
    DiagArgs a{};
    a.t = c->f[ATJUP_F_T]; a.u = c->f[ATJUP_F_U]; a.v = c->f[ATJUP_F_V]; a.w = c->f[ATJUP_F_W];
    a.p_dyn = c->f[ATJUP_F_P_DYN]; a.p_stat = c->f[ATJUP_F_P_STAT];
    a.h2o = c->f[ATJUP_F_H2O]; a.nh3 = c->f[ATJUP_F_NH3];
    a.solid = c->solid; a.rad = c->rad; a.sin_the = c->sin_the; a.geo = c->geo;
    a.cor = c->f[ATJUP_F_CORIOLIS_FORCE]; a.cen = c->f[ATJUP_F_CENTRIFUGAL_FORCE];
    a.buo = c->f[ATJUP_F_BUOYANCY_FORCE]; a.pgf = c->f[ATJUP_F_PRESGRAD_FORCE];
    a.ql = c->f[ATJUP_F_Q_LATENT]; a.qs = c->f[ATJUP_F_Q_SENSIBLE];
    for (int q = 0; q < 8; q++) a.cc[q] = mc.cc[q];
    a.ep_w = mc.gas[ATJUP_GAS_H2O].ep; a.lv_w = mc.gas[ATJUP_GAS_H2O].lv; a.ls_w = mc.gas[ATJUP_GAS_H2O].ls;
    a.ep_a = mc.gas[ATJUP_GAS_NH3].ep; a.lv_a = mc.gas[ATJUP_GAS_NH3].lv; a.ls_a = mc.gas[ATJUP_GAS_NH3].ls;
    a.fix_lat = mc.qheat_scale ? (P.im - 1) / 1.0e3 : 1.0;
    a.fix_sen = mc.qheat_scale ? P.L_atm * (P.im - 1) * (P.im - 1) / 1.0e3 : 1.0;
    a.omega = P.omega; a.Coriolis = P.Coriolis; a.centrifugal = P.centrifugal;
    a.buoyancy = P.buoyancy; a.r_mix = P.r_mix; a.R_mix = P.R_mix; a.g = P.g; a.t_ref = P.t_ref;
    a.p_dyn_to_bar = P.p_dyn_to_bar; a.L_atm = P.L_atm; a.u_0 = P.u_0; a.cp_mix = P.cp_mix;
    a.dr = P.dr; a.dthe = P.dthe; a.dphi = P.dphi;
    a.im = P.im; a.jm = P.jm; a.km = P.km; a.KP = c->KP; a.costhe_abs = mc.costhe_abs;
    return a;
}

MicroArgs make_args(AtjupCtx* c) {
    const AtjupParams& P = c->P;
    MicroArgs a{};
    a.t = c->f[ATJUP_F_T];
    a.p_stat = c->f[ATJUP_F_P_STAT];
    a.rho_mix = c->f[ATJUP_F_RHO_MIX];
    a.u = c->f[ATJUP_F_U];
    a.v = c->f[ATJUP_F_V];
    a.w = c->f[ATJUP_F_W];
    for (int s = 0; s < ATJUP_S_COUNT; s++) a.q[s] = c->f[kScalarField[s]];
    const int sp[9] = {ATJUP_F_S_PRECIP_H2O, ATJUP_F_S_PRECIP_H2O_CLOUD, ATJUP_F_S_PRECIP_H2O_ICE,
                       ATJUP_F_S_PRECIP_NH3, ATJUP_F_S_PRECIP_NH3_CLOUD, ATJUP_F_S_PRECIP_NH3_ICE,
                       ATJUP_F_S_PRECIP_CH4, ATJUP_F_S_PRECIP_CH4_CLOUD, ATJUP_F_S_PRECIP_CH4_ICE};
    for (int q = 0; q < 9; q++) a.sprec[q] = c->f[sp[q]];
    a.Q_rad = c->f[ATJUP_F_Q_RAD];
    a.Q_precip = c->f[ATJUP_F_Q_PRECIP];
    a.difflux[0] = c->f[ATJUP_F_DIFFLUX_H2S];
    a.difflux[1] = c->f[ATJUP_F_DIFFLUX_NH3];
    a.difflux[2] = c->f[ATJUP_F_DIFFLUX_NH4SH];
    a.massflux[0] = c->f[ATJUP_F_MASSFLUX_H2S];
    a.massflux[1] = c->f[ATJUP_F_MASSFLUX_NH3];
    a.massflux[2] = c->f[ATJUP_F_MASSFLUX_NH4SH];
    a.fluxlim = c->f[ATJUP_F_FLUXLIM_NH4SH];
    a.topo = c->topo;
    a.layer_h = c->layer_h;
    a.solid = c->solid;
    a.rad = c->rad;
    a.sin_the = c->sin_the;
    a.cos_lat = c->cos_lat;
    a.geo = c->geo;
    a.mc = c->micro;
    a.im = P.im; a.jm = P.jm; a.km = P.km; a.KP = c->KP; a.local_rho = P.local_rho;
    a.t_ref = P.t_ref; a.g = P.g; a.r_mix = P.r_mix; a.cp_mix = P.cp_mix; a.L_atm = P.L_atm;
    a.u_0 = P.u_0; a.dr = P.dr; a.dthe = P.dthe; a.dphi = P.dphi;
    return a;
}

}  // namespace

int launch_micro(AtjupCtx* c, int what) {
    const AtjupParams& P = c->P;
    if (P.im > MAX_IM) {
        set_error("microphysics: more than 64 radial levels");
        return ATJUP_ERR_UNSUPPORTED;
    }
    MicroArgs a = make_args(c);
    const int TB = 128;
    const dim3 gcol((P.km + TB - 1) / TB, P.jm);
    const dim3 gcell((P.km + TB - 1) / TB, P.jm, P.im);
    switch (what) {
    case MICRO_RADIATION:
        radiation_kernel<<<gcol, TB, 0, c->stream>>>(a);
        c->launches++;
        break;
    case MICRO_PRECIP:
        precip_kernel<<<dim3((P.km + PR_COLS - 1) / PR_COLS, P.jm), dim3(PR_COLS, 3), 0, c->stream>>>(a);
        c->launches++;
        break;
    case MICRO_NH4SH:
        nh4sh_kernel<<<gcell, TB, 0, c->stream>>>(a, 4705.0 * std::log(10.0) * 8314.46 / 51.1114);
        c->launches++;
        break;
    case MICRO_CHEMISTRY: {
        int rc;
        difflux_kernel<<<gcell, TB, 0, c->stream>>>(a);
        c->launches++;
        ATJUP_CHECK_LAUNCH("difflux_kernel");
        for (int q = 0; q < 3; q++)
            if ((rc = launch_shapiro(c, a.difflux[q], 2, 1.0, 1, 1))) return rc;
        massflux_kernel<<<gcell, TB, 0, c->stream>>>(a);
        fluxlim_kernel<<<gcell, TB, 0, c->stream>>>(a);
        c->launches += 2;
        ATJUP_CHECK_LAUNCH("massflux/fluxlim kernels");
        for (int q = 0; q < 3; q++)
            if ((rc = launch_shapiro(c, a.massflux[q], 2, 1.0, 1, 1))) return rc;
        if ((rc = launch_shapiro(c, a.fluxlim, 2, 1.0, 1, 1))) return rc;
        break;
    }
    case MICRO_CLAMP:
        clamp_species_kernel<<<gcell, TB, 0, c->stream>>>(a);
        c->launches++;
        break;
    case MICRO_DIAG:
        diagnostics_kernel<<<gcell, TB, 0, c->stream>>>(diag_args(c));
        c->launches++;
        break;
    default:
        set_error("microphysics: unknown routine");
        return ATJUP_ERR_ARG;
    }
    ATJUP_CHECK_LAUNCH("microphysics");
    return ATJUP_OK;
}

}  // namespace atjup
