// The turbulence closure update between steps: Turbulence<cJupiterModel>::run
// (Turbulence.h:307-328) and the driver's turbWallOmega (cJupiterModel.cpp:360-377).
//
//   vel_star_kernel    compute_vel_star (336-360): friction velocity per column
//   clamp_in_kernel    the first clamp pass of compute_sources (624-626, 634-639)
//   sources_kernel     production with curvature terms and the model routine per cell
//                      (655-867, 886-1106): nue, prod, tke_source, dis_source
//   clamp_out_kernel   the second clamp pass (627-633, 870-880)
//   column_kernel      apply_wall_bc (383-422), zero_land_cells (592-610), clamp_nue (565-588)
//   seam / lid / pole  seam_copy (543-559), fill_lid_corners (511-536)
//   wall_omega_kernel  turbWallOmega
//
// Every pass is one thread per cell or per column with k fastest; the sources kernel reads the
// 7-point stencils of u, v, w, k*, omega* (k neighbours from the warp's own loads, i and j
// neighbours from L2) and writes four fields. The clamp passes are separate kernels because the
// reference runs them as separate sweeps: a cell's sources read its neighbours' clamped k*,
// omega*, and the second clamp must not change a value a neighbour still has to read.
#include "ctx.cuh"

namespace atjup {
namespace {

enum : uint8_t { NB_S = 1, NB_IP = 2, NB_IM = 4, NB_JP = 8, NB_JM = 16, NB_KP = 32, NB_KM = 64 };

struct TurbArgs {
    const double *u, *v, *w, *t;
    double *tke, *dis, *tken, *disn, *nue, *prod, *tke_source, *dis_source;
    double* vel_star;              // [jm][KP]
    const uint8_t* flags;
    const GeoIJ* geo;
    const double* sin_the;         // [jm] sin(the_j)
    const double* rad;             // [im]
    const int32_t* topo;           // [jm * km]
    const float* layer_h;          // [im]
    int im, jm, km, KP, model, turb_free, turb_curv, turb_buoy, abl_taper, wall_omega;
    double dr, dthe, dphi, u_0, L_m, nue_max, t_ref, g, cp_mix, re_turb;
    double k_bg_free, vel_star_max, abl_height, taper_dz;
    int wall_only;                 // column_kernel: the wall law alone (the loop's wall hold)
};

__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double clamp3(double x, double lo, double hi) {
    return (x < lo) ? lo : ((x > hi) ? hi : x);
}
__device__ __forceinline__ double height_m(const TurbArgs& a, int i) {
    return ((i < 0 || i > a.im - 1) ? (double)(-1.0f) : (double)a.layer_h[i]) * 1.0e3;
}
__device__ __forceinline__ double layer_dz_m(const TurbArgs& a, int i) {
    if (i < 0 || i > a.im - 2) return -1.0;
    return (double)(a.layer_h[i + 1] - a.layer_h[i]) * 1.0e3;
}

constexpr double C_NUE = 0.028, DIS_MIN = 1.0e-10, NUE_AIR = 1.8e-5;

// ---- compute_vel_star: one thread per (j, k) ----
__global__ void vel_star_kernel(TurbArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= a.km) return;
    double vs = 0.05;
    if (!a.turb_free) {
        int is = a.topo[(size_t)j * a.km + k] + 1;
        if (is > a.im - 1) is = a.im - 1;
        const size_t c = ((size_t)is * a.jm + j) * a.KP + k;
        const double vw2 = a.v[c] * a.v[c] + a.w[c] * a.w[c];
        if (isfinite(vw2)) vs = clamp3(sqrt(0.002) * (a.u_0 * sqrt(vw2)), 0.05, a.vel_star_max);
    }
    a.vel_star[(size_t)j * a.KP + k] = vs;
}

// interior region of compute_sources: i in [1, im-2], j in [1, jm-2], k in [0, km-2], fluid
__device__ __forceinline__ bool source_cell(const TurbArgs& a, int i, int j, int k, size_t& c) {
    if (k > a.km - 2 || j < 1 || j > a.jm - 2 || i < 1 || i > a.im - 2) return false;
    c = ((size_t)i * a.jm + j) * a.KP + k;
    return !(a.flags[c] & NB_S);
}

__global__ void clamp_in_kernel(TurbArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    size_t c;
    if (!source_cell(a, i, j, k, c)) return;
    a.tke[c] = dmax(0.0, a.tke[c]);
    a.dis[c] = dmax(DIS_MIN, a.dis[c]);
}

__global__ void __launch_bounds__(128) sources_kernel(TurbArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    size_t c;
    if (!source_cell(a, i, j, k, c)) return;
    const uint8_t fl = a.flags[c];
    const size_t plane = (size_t)a.jm * a.KP;
    const size_t row = c - k;
    const int ke = (k >= a.km - 2) ? 0 : k + 1, kw = (k == 0) ? a.km - 2 : k - 1;
    const size_t cip = c + plane, cim = c - plane, cjp = c + a.KP, cjm = c - a.KP;
    const size_t ckp = row + ke, ckm = row + kw;
    const double rm = a.rad[i];
    double sinthe = a.sin_the[j];
    if (sinthe == 0.0) sinthe = 1.0e-5;
    const double costhe = a.geo[(size_t)i * a.jm + j].costhe;
    const double cotanthe = costhe / sinthe;
    const double inv_rm = 1.0 / rm;
    const double rmsinthe = rm * sinthe;
    const double inv_2dr = 1.0 / (2.0 * a.dr);
    const double inv_2dthe = 1.0 / (2.0 * a.dthe);
    const double inv_2dphi = 1.0 / (2.0 * a.dphi);
    const double inv_rm2dthe = inv_2dthe / rm;
    const double inv_rmsinthe2dphi = inv_2dphi / rmsinthe;
    const double *U = a.u, *V = a.v, *W = a.w;
    const double dudr = (U[cip] - U[cim]) * inv_2dr, dvdr = (V[cip] - V[cim]) * inv_2dr;
    const double dwdr = (W[cip] - W[cim]) * inv_2dr;
    const double dudthe = (U[cjp] - U[cjm]) * inv_rm2dthe, dvdthe = (V[cjp] - V[cjm]) * inv_rm2dthe;
    const double dwdthe = (W[cjp] - W[cjm]) * inv_rm2dthe;
    const double dudphi = (U[ckp] - U[ckm]) * inv_rmsinthe2dphi;
    const double dvdphi = (V[ckp] - V[ckm]) * inv_rmsinthe2dphi;
    const double dwdphi = (W[ckp] - W[ckm]) * inv_rmsinthe2dphi;

    const double *TK = a.tke, *DS = a.dis;
    const double tk0 = TK[c], ds0 = DS[c];
    const bool nb = fl & NB_IM, njm = fl & NB_JM, njp = fl & NB_JP, nkm = fl & NB_KM, nkp = fl & NB_KP;
    const double tke_im1 = nb ? tk0 : TK[cim], dis_im1 = nb ? ds0 : DS[cim];
    const double tke_jm1 = njm ? tk0 : TK[cjm], tke_jp1 = njp ? tk0 : TK[cjp];
    const double dis_jm1 = njm ? ds0 : DS[cjm], dis_jp1 = njp ? ds0 : DS[cjp];
    const double tke_km1 = nkm ? tk0 : TK[ckm], tke_kp1 = nkp ? tk0 : TK[ckp];
    const double dis_km1 = nkm ? ds0 : DS[ckm], dis_kp1 = nkp ? ds0 : DS[ckp];
    const double tk_ip = TK[cip], ds_ip = DS[cip];
    const double dtkedr = (tk_ip - tke_im1) * inv_2dr;
    const double ddisdr = (ds_ip - dis_im1) * inv_2dr;

    double cnue;
    {
        const double dis_here = dmax(ds0, DIS_MIN);
        const double tke_here = dmax(tk0, 0.0);
        cnue = (a.model == ATJUP_TURB_K_EPSILON) ? C_NUE * tke_here * tke_here / dis_here
                                                 : tke_here / dis_here;
        cnue = dmin(cnue, a.nue_max);
    }
    const double u_r = a.turb_curv ? U[c] * inv_rm : 0.0;
    const double v_r = a.turb_curv ? V[c] * inv_rm : 0.0;
    const double w_r = a.turb_curv ? W[c] * inv_rm : 0.0;
    const double v_cot_r = v_r * cotanthe, w_cot_r = w_r * cotanthe;
    const double g_rr = dudr, g_rt = dudthe - v_r, g_rp = dudphi - w_r;
    const double g_tr = dvdr, g_tt = dvdthe + u_r, g_tp = dvdphi - w_cot_r;
    const double g_pr = dwdr, g_pt = dwdthe, g_pp = dwdphi + u_r + v_cot_r;
    const double der = 0.66667 * (g_rr + g_tt + g_pp);
    const double prod = dmax(0.0,
          (cnue * (2.0 * g_rr - der) - 0.66667 * tk0) * g_rr
        + (cnue * (g_rt + g_tr)) * g_rt
        + (cnue * (g_rp + g_pr)) * g_rp
        + (cnue * (2.0 * g_tt - der) - 0.66667 * tk0) * g_tt
        + (cnue * (g_tr + g_rt)) * g_tr
        + (cnue * (g_tp + g_pt)) * g_tp
        + (cnue * (2.0 * g_pp - der) - 0.66667 * tk0) * g_pp
        + (cnue * (g_pr + g_rp)) * g_pr
        + (cnue * (g_pt + g_tp)) * g_pt);
    const double W12 = g_rt - g_tr, W13 = g_rp - g_pr, W23 = g_tp - g_pt;
    const double Omega = sqrt(W12 * W12 + W13 * W13 + W23 * W23);
    const double L_m = a.L_m;
    const double y_mount = height_m(a, a.topo[(size_t)j * a.km + k]);

    double nue, tsrc, dsrc;
    if (a.model == ATJUP_TURB_K_EPSILON) {                          // Turbulence.h:886-927
        const double C_eps_1 = 1.35, C_eps_2 = 1.80;
        const double y_phys = a.turb_free ? 1.0e20 : dmax(height_m(a, i) - y_mount, L_m);
        const double y_star = y_phys / L_m;
        nue = C_NUE * tk0 * tk0 / dmax(ds0, DIS_MIN);
        const double d_plus = y_phys * a.vel_star[(size_t)j * a.KP + k] / NUE_AIR;
        const double f_nue = 1.0 - exp(-0.0115 * d_plus);
        const double Re_T = tk0 * tk0 * a.u_0 * L_m / dmax(ds0 * NUE_AIR, DIS_MIN * NUE_AIR);
        const double f_2 = 1.0 - 0.4 / 1.8 * exp(-Re_T * Re_T / 36.0);
        nue *= f_nue;
        const double y_star2 = y_star * y_star;
        const double L_k = -2.0 * tk0 / y_star2;
        const double L_w = -2.0 * ds0 / y_star2 * exp(-d_plus / 2.0);
        const double tke_safe = dmax(tk0, DIS_MIN);
        const double P_w = C_eps_1 * ds0 / tke_safe * prod;
        const double Y_w = C_eps_2 * f_2 * ds0 * ds0 / tke_safe;
        tsrc = prod - ds0 + L_k / a.re_turb;
        dsrc = P_w - Y_w + L_w / a.re_turb;
    } else {
        const double exp_rm_k = 1.0 / (rm + 1.0);
        const double dtkedr_neu = nb ? (tk_ip - tk0) * (1.0 / (2.0 * a.dr)) * exp_rm_k : dtkedr;
        const double ddisdr_neu = nb ? (ds_ip - ds0) * (1.0 / (2.0 * a.dr)) * exp_rm_k : ddisdr;
        const double dtkedthe_neu = (tke_jp1 - tke_jm1) / (rm * 2.0 * a.dthe);
        const double ddisdthe_neu = (dis_jp1 - dis_jm1) / (rm * 2.0 * a.dthe);
        const double dtkedphi_neu = (tke_kp1 - tke_km1) / (rmsinthe * 2.0 * a.dphi);
        const double ddisdphi_neu = (dis_kp1 - dis_km1) / (rmsinthe * 2.0 * a.dphi);
        const double grad_dot = dtkedr_neu * ddisdr_neu + dtkedthe_neu * ddisdthe_neu +
                                dtkedphi_neu * ddisdphi_neu;
        if (a.model == ATJUP_TURB_K_OMEGA) {                        // Turbulence.h:930-1017
            const double bet_star = 0.09, gam = 0.52, C_lim = 0.875, bet_0 = 0.0708;
            const double dudr_k = (U[cip] - U[cim]) / (2.0 * a.dr) / (rm + 1.0);
            const double dvdthe_k = (V[cjp] - V[cjm]) / (rm * 2.0 * a.dthe);
            const double dwdphi_k = (W[ckp] - W[ckm]) / (rmsinthe * 2.0 * a.dphi);
            const double dudthe_u = (U[cjp] - U[cjm]) / (rm * 2.0 * a.dthe);
            const double dudphi_u = (U[ckp] - U[ckm]) / (rmsinthe * 2.0 * a.dphi);
            const double dvdr_u = (V[cip] - V[cim]) / (2.0 * a.dr) / (rm + 1.0);
            const double dwdr_u = (W[cip] - W[cim]) / (2.0 * a.dr) / (rm + 1.0);
            const double dvdphi_u = (V[ckp] - V[ckm]) / (rmsinthe * 2.0 * a.dphi);
            const double dwdthe_u = (W[cjp] - W[cjm]) / (rm * 2.0 * a.dthe);
            const double S11 = dudr_k, S22 = dvdthe_k, S33 = dwdphi_k;
            const double S12 = 0.5 * (dudthe_u + dvdr_u);
            const double S13 = 0.5 * (dudphi_u + dwdr_u);
            const double S23 = 0.5 * (dvdphi_u + dwdthe_u);
            const double S_mag = sqrt(2.0 * (S11 * S11 + S22 * S22 + S33 * S33 +
                                             2.0 * (S12 * S12 + S13 * S13 + S23 * S23)));
            const double w_hat = dmax(ds0, C_lim * S_mag / sqrt(bet_star));
            const double sig_d = (grad_dot <= 0.0) ? 0.0 : 0.125;
            const double bd = bet_star * dmax(ds0, 1.0e-20);
            const double chi_w = fabs(Omega * Omega * S_mag / (bd * bd * bd));   // pow(bd, 3)
            const double f_bet = (1.0 + 85.0 * chi_w) / (1.0 + 100.0 * chi_w);
            const double bet_wc = bet_0 * f_bet;
            nue = tk0 / dmax(w_hat, 1.0e-20);
            const double P_k = dmin(prod, 20.0 * bet_star * tk0 * ds0);
            const double Y_k = bet_star * tk0 * ds0;
            const double P_w = gam * ds0 / dmax(tk0, 1.0e-20) * P_k;
            const double Y_w = bet_wc * ds0 * ds0;
            const double D_w = sig_d / dmax(ds0, 1.0e-20) * grad_dot;
            tsrc = P_k - Y_k;
            dsrc = P_w - Y_w + D_w;
        } else {                                                    // Turbulence.h:1021-1106
            const double a1 = 0.31, bet_star = 0.09, bet1 = 0.0333, bet2 = 0.0368;
            const double gam1 = 0.413, gam2 = 0.2, sig_w2 = 1.168;
            const double nue_air_nd = NUE_AIR / (a.u_0 * L_m);
            const double dz_layer = dmax(1.0, layer_dz_m(a, i - 1 > 0 ? i - 1 : 0));
            const double y_phys = a.turb_free ? 1.0e20 : dmax(height_m(a, i) - y_mount, dz_layer);
            const double y_star = y_phys / L_m;
            const double CD_kw = dmax(2.0 * sig_w2 / dmax(ds0, 1.0e-20) * grad_dot, 1.0e-20);
            const double dis_safe = dmax(ds0, 1.0e-20);
            const double arg1 = dmin(dmax(sqrt(tk0) / (bet_star * dis_safe * y_star),
                                          500.0 * nue_air_nd / (y_star * y_star * dis_safe)),
                                     4.0 * sig_w2 * tk0 / (CD_kw * y_star * y_star));
            const double arg2 = dmax(2.0 * sqrt(tk0) / (bet_star * dis_safe * y_star),
                                     500.0 * nue_air_nd / (y_star * y_star * dis_safe));
            const double a1sq = arg1 * arg1;
            const double F1 = tanh(a1sq * a1sq);                                // pow(arg1, 4)
            const double F2 = tanh(arg2 * arg2);                                // pow(arg2, 2)
            nue = a1 * tk0 / dmax(a1 * dis_safe, Omega * F2);
            const double tke_safe = dmax(tk0, 1.0e-20);
            const double P_k = dmin(prod, 20.0 * bet_star * tke_safe * dis_safe);
            const double Y_k = bet_star * tke_safe * dis_safe;
            const double P_w = (F1 * gam1 + (1.0 - F1) * gam2) * P_k * dis_safe / tke_safe;
            const double Y_w = (F1 * bet1 + (1.0 - F1) * bet2) * dis_safe * dis_safe;
            const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_safe * grad_dot;
            tsrc = P_k - Y_k;
            dsrc = P_w - Y_w + D_w;
        }
    }
    if (a.turb_buoy != 0) {                                         // Turbulence.h:843-867
        const double T = a.t[c] * a.t_ref;
        const double dz = height_m(a, i + 1) - height_m(a, i - 1);
        const double dTdz = (a.t[cip] - a.t[cim]) * a.t_ref / dz;
        const double Gam = a.g / a.cp_mix;
        const double N2 = (T > 0.0 && dz > 0.0) ? a.g / T * (dTdz + Gam) * 1.0 : 0.0;
        if (isfinite(N2) && (N2 > 0.0 || a.turb_buoy == 2)) {
            const double tL = L_m / a.u_0;
            tsrc -= dmax(0.0, nue) * N2 * tL * tL / 0.9;
        }
    }
    a.prod[c] = prod;
    a.nue[c] = nue;
    a.tke_source[c] = tsrc;
    a.dis_source[c] = dsrc;
}

__global__ void clamp_out_kernel(TurbArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    size_t c;
    if (!source_cell(a, i, j, k, c)) return;
    double k_bg_nd;
    if (a.turb_free) {
        k_bg_nd = a.k_bg_free;
    } else {
        const double vs = a.vel_star[(size_t)j * a.KP + k];
        k_bg_nd = 0.01 * vs * vs / (sqrt(C_NUE) * a.u_0 * a.u_0);
    }
    const double tk = dmax(k_bg_nd, a.tke[c]);
    const double ds = dmax(DIS_MIN, a.dis[c]);
    a.tke[c] = tk;
    a.dis[c] = ds;
    a.nue[c] = clamp3(a.nue[c], 0.0, a.nue_max);
    const double dis_src_max = 20.0 * ds * ds;
    a.dis_source[c] = clamp3(a.dis_source[c], -dis_src_max, dis_src_max);
    const double tke_src_max = 20.0 * tk * ds;
    a.tke_source[c] = clamp3(a.tke_source[c], -tke_src_max, tke_src_max);
}

// apply_wall_bc, zero_land_cells and clamp_nue: one thread per (j, k) column
__global__ void column_kernel(TurbArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (k >= a.km) return;
    const size_t plane = (size_t)a.jm * a.KP;
    const size_t c0 = (size_t)j * a.KP + k;     // cell (0, j, k)
    const int i_w = a.topo[(size_t)j * a.km + k];
    if (!a.turb_free && i_w > 0 && i_w < a.im - 1) {
        const double y1 = dmax(layer_dz_m(a, i_w - 1 > 0 ? i_w - 1 : 0), 1.0);
        const double vs = a.vel_star[(size_t)j * a.KP + k];
        const double nd_omega = a.L_m / a.u_0;
        const size_t cw = c0 + (size_t)i_w * plane;
        a.tke[cw] = vs * vs / (sqrt(C_NUE) * a.u_0 * a.u_0);
        a.nue[cw] = 0.0;
        if (a.model == ATJUP_TURB_K_EPSILON) a.dis[cw] = 0.0;
        else if (a.model == ATJUP_TURB_K_OMEGA) a.dis[cw] = 6.0 * NUE_AIR / (0.075 * y1 * y1) * nd_omega;
        else a.dis[cw] = 60.0 * NUE_AIR / (0.0333 * y1 * y1) * nd_omega;
    } else {
        a.tke[c0] = a.tke[c0 + plane];
        a.dis[c0] = a.dis[c0 + plane];
        a.nue[c0] = a.nue[c0 + plane];
    }
    if (a.wall_only) return;
    const double y_surf = height_m(a, i_w);
    for (int i = 0; i < a.im; i++) {
        const size_t c = c0 + (size_t)i * plane;
        if (a.flags[c] & NB_S) {
            a.tke[c] = 0.0; a.tken[c] = 0.0; a.dis[c] = 0.0; a.disn[c] = 0.0;
            a.nue[c] = 0.0; a.prod[c] = 0.0; a.tke_source[c] = 0.0; a.dis_source[c] = 0.0;
        }
        double f = 1.0;
        if (a.abl_taper) {
            const double z_agl = height_m(a, i) - y_surf;
            f = clamp3((a.abl_height + a.taper_dz - z_agl) / a.taper_dz, 0.0, 1.0);
        }
        a.nue[c] = clamp3(a.nue[c], 0.0, a.nue_max) * f;
    }
}

__device__ __forceinline__ void copy8(const TurbArgs& a, size_t dst, size_t src) {
    a.tke[dst] = a.tke[src]; a.dis[dst] = a.dis[src]; a.tken[dst] = a.tken[src];
    a.disn[dst] = a.disn[src]; a.nue[dst] = a.nue[src]; a.prod[dst] = a.prod[src];
    a.tke_source[dst] = a.tke_source[src]; a.dis_source[dst] = a.dis_source[src];
}

// seam_copy: one thread per (i, j) row
__global__ void seam_kernel(TurbArgs a) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= a.jm) return;
    const size_t row = ((size_t)i * a.jm + j) * a.KP;
    copy8(a, row + a.km - 1, row);
}

// fill_lid_corners, TURB_FREE branch: lid plane from the plane below (j in [1, jm-2])
__global__ void lid_kernel(TurbArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y + 1;
    if (k >= a.km || j > a.jm - 2) return;
    const size_t dst = ((size_t)(a.im - 1) * a.jm + j) * a.KP + k;
    copy8(a, dst, dst - (size_t)a.jm * a.KP);
}

// then the pole rows of every plane from their neighbours
__global__ void pole_kernel(TurbArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (k >= a.km) return;
    const size_t base = (size_t)i * a.jm * a.KP + k;
    copy8(a, base, base + a.KP);
    copy8(a, base + (size_t)(a.jm - 1) * a.KP, base + (size_t)(a.jm - 2) * a.KP);
}

// turbWallOmega (cJupiterModel.cpp:360-377)
__global__ void wall_omega_kernel(TurbArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (k >= a.km) return;
    const int i_w = a.topo[(size_t)j * a.km + k];
    if (i_w <= 0 || i_w >= a.im - 1) return;
    const double bet_star = 0.09, bet_1 = 0.0333, kappa = 0.41;
    const double y1 = dmax(layer_dz_m(a, i_w - 1 > 0 ? i_w - 1 : 0), 1.0);
    const double y = 0.5 * y1;
    const double om_vis = 60.0 * NUE_AIR / (bet_1 * y1 * y1);
    const double om_log = a.vel_star[(size_t)j * a.KP + k] / (sqrt(bet_star) * kappa * y);
    a.dis[((size_t)i_w * a.jm + j) * a.KP + k] = sqrt(om_vis * om_vis + om_log * om_log) * (a.L_m / a.u_0);
}

}  // namespace

namespace {
TurbArgs turb_args(AtjupCtx* c);
}

int launch_turbulence(AtjupCtx* c) {
    const AtjupParams& P = c->P;
    const AtjupPhysics& H = c->phys;
    TurbArgs a = turb_args(c);
    const int TB = 128;
    const dim3 bcol((P.km + TB - 1) / TB, P.jm);
    const dim3 bcell((P.km + TB - 1) / TB, P.jm, P.im);
    vel_star_kernel<<<bcol, TB, 0, c->stream>>>(a);
    clamp_in_kernel<<<bcell, TB, 0, c->stream>>>(a);
    sources_kernel<<<bcell, TB, 0, c->stream>>>(a);
    clamp_out_kernel<<<bcell, TB, 0, c->stream>>>(a);
    column_kernel<<<bcol, TB, 0, c->stream>>>(a);
    seam_kernel<<<dim3((P.jm + TB - 1) / TB, P.im), TB, 0, c->stream>>>(a);
    c->launches += 6;
    if (H.turb_free) {
        lid_kernel<<<dim3((P.km + TB - 1) / TB, P.jm - 2), TB, 0, c->stream>>>(a);
        pole_kernel<<<dim3((P.km + TB - 1) / TB, P.im), TB, 0, c->stream>>>(a);
        c->launches += 2;
    }
    if (H.turb_wall_omega != 0 && H.turb_model != ATJUP_TURB_K_EPSILON) {
        wall_omega_kernel<<<bcol, TB, 0, c->stream>>>(a);
        c->launches++;
    }
    ATJUP_CHECK_LAUNCH("turbulence kernels");
    return ATJUP_OK;
}

// The loop's wall hold after the boundary passes (ATJUP_TURB_WALL_HOLD 1, cJupiterModel.cpp:
// 1274-1280): apply_wall_bc and turbWallOmega again.
int launch_turb_wall_hold(AtjupCtx* c) {
    const AtjupParams& P = c->P;
    const AtjupPhysics& H = c->phys;
    TurbArgs a = turb_args(c);
    a.wall_only = 1;
    const int TB = 128;
    const dim3 bcol((P.km + TB - 1) / TB, P.jm);
    column_kernel<<<bcol, TB, 0, c->stream>>>(a);
    c->launches++;
    if (H.turb_wall_omega != 0 && H.turb_model != ATJUP_TURB_K_EPSILON) {
        wall_omega_kernel<<<bcol, TB, 0, c->stream>>>(a);
        c->launches++;
    }
    ATJUP_CHECK_LAUNCH("turbulence wall hold");
    return ATJUP_OK;
}

namespace {
TurbArgs turb_args(AtjupCtx* c) {
    const AtjupParams& P = c->P;
    const AtjupPhysics& H = c->phys;
    TurbArgs a{};
    a.u = c->f[ATJUP_F_U]; a.v = c->f[ATJUP_F_V]; a.w = c->f[ATJUP_F_W]; a.t = c->f[ATJUP_F_T];
    a.tke = c->f[ATJUP_F_TKE]; a.dis = c->f[ATJUP_F_DIS];
    a.tken = c->fn[ATJUP_F_TKE]; a.disn = c->fn[ATJUP_F_DIS];
    a.nue = c->f[ATJUP_F_NUE]; a.prod = c->f[ATJUP_F_PROD];
    a.tke_source = c->f[ATJUP_F_TKE_SOURCE]; a.dis_source = c->f[ATJUP_F_DIS_SOURCE];
    a.vel_star = c->f2[ATJUP_F2_VEL_STAR];
    a.flags = c->nbflags; a.geo = c->geo; a.sin_the = c->sin_the; a.rad = c->rad;
    a.topo = c->topo; a.layer_h = c->layer_h;
    a.im = P.im; a.jm = P.jm; a.km = P.km; a.KP = c->KP;
    a.model = H.turb_model; a.turb_free = H.turb_free; a.turb_curv = H.turb_curv;
    a.turb_buoy = H.turb_buoy; a.abl_taper = H.abl_taper; a.wall_omega = H.turb_wall_omega;
    a.dr = P.dr; a.dthe = P.dthe; a.dphi = P.dphi; a.u_0 = P.u_0;
    a.L_m = P.L_atm * 1.0e3;
    a.nue_max = H.nue_max_phys / (P.u_0 * a.L_m);
    a.t_ref = P.t_ref; a.g = P.g; a.cp_mix = P.cp_mix; a.re_turb = H.re_turb;
    a.k_bg_free = H.turb_k_bg / (P.u_0 * P.u_0);
    a.vel_star_max = H.vel_star_max;
    a.abl_height = H.abl_height;
    a.taper_dz = c->turb_taper_dz;
    return a;
}
}  // namespace

}  // namespace atjup
