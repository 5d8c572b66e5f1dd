/*
 * CPU oracle for the ATJUP hot path -- TEST INFRASTRUCTURE ONLY (see atjup_oracle.h).
 *
 * Each routine restates one reference routine; the file:line it follows is given at the routine.
 * Expressions keep the reference's operand order so that, built with FMA contraction off, the
 * FP64 results are bit-identical to the reference's own -- that is what lets tests pin this file
 * to the reference exactly rather than to a tolerance.
 */
#include "atjup_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, k) (((size_t)(i) * (size_t)jm + (size_t)(j)) * (size_t)km + (size_t)(k))
#define C43 (4.0 / 3.0)
#define C13 (1.0 / 3.0)

static inline int phi_wrap(int periodic, int kk, int km) {
    /* ATPhys.h:131-135: the ring of km-1 distinct meridians */
    if (!periodic) return kk;
    const int n = km - 1;
    return kk < 0 ? kk + n : (kk >= n ? kk - n : kk);
}

static inline double dmax(double a, double b) { return a < b ? b : a; }   /* std::max(a, b) */
static inline double dmin(double a, double b) { return b < a ? b : a; }   /* std::min(a, b) */

/* The bit pattern test of RungeKutta_Jup_Turb.cpp:273-278: NaN or +-Inf -> lo. */
static double safe_clamp(double v, double lo, double hi) {
    uint64_t bits;
    memcpy(&bits, &v, sizeof bits);
    if ((bits & 0x7FF0000000000000ULL) == 0x7FF0000000000000ULL) return lo;
    return (v < lo) ? lo : ((v > hi) ? hi : v);
}

/* Geometry of one (i, j) row, built as RungeKutta_Jup_Turb.cpp:388-411 builds CellGeometry. */
typedef struct {
    double rm, rm2, exp_rm, exp_2_rm, sinthe, sinthe2, costhe, cotanthe;
    double inv_rm, inv_rm2, inv_rmsinthe, inv_rm2sinthe, inv_rm2sinthe2, costhe_inv_rm2sinthe;
    double inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
} geom;

static void make_geom(const AtjupParams* P, const ora_grid* G, int i, int j, geom* g) {
    g->rm = G->rad[i];
    g->rm2 = g->rm * g->rm;
    g->exp_rm = 1.0;                         /* coord_stretching = false (param.py:52)      */
    g->exp_2_rm = g->exp_rm * g->exp_rm;
    g->sinthe = dmax(P->sinthe_min, fabs(sin(G->the[j])));
    g->sinthe2 = g->sinthe * g->sinthe;
    g->costhe = cos(G->the[j]);
    g->cotanthe = g->costhe / g->sinthe;
    g->inv_rm = 1.0 / g->rm;
    g->inv_rm2 = 1.0 / g->rm2;
    g->inv_rmsinthe = 1.0 / (g->rm * g->sinthe);
    g->inv_rm2sinthe = g->inv_rm2 / g->sinthe;
    g->inv_rm2sinthe2 = g->inv_rm2 / g->sinthe2;
    g->costhe_inv_rm2sinthe = g->costhe * g->inv_rm2sinthe;
    g->inv_2dr = 1.0 / (2.0 * P->dr);
    g->inv_2dthe = 1.0 / (2.0 * P->dthe);
    g->inv_2dphi = 1.0 / (2.0 * P->dphi);
    g->inv_dr2 = 1.0 / (P->dr * P->dr);
    g->inv_dthe2 = 1.0 / (P->dthe * P->dthe);
    g->inv_dphi2 = 1.0 / (P->dphi * P->dphi);
}

/* ------------------------------------------------------------------------------------------ */
/* RungeKutta_Jup_Turb.cpp:47-69 -- sin(theta)-weighted level mean of g p_stat / (r R T t_ref)  */
void ora_buoy_ref_level(const AtjupParams* P, const ora_grid* G, ora_state* S) {
    const int im = P->im, jm = P->jm, km = P->km;
    for (int i = 0; i < im; i++) {
        double sum = 0.0, wsum = 0.0;
        for (int j = 0; j < jm; j++) {
            const double wgt = sin(G->the[j]);
            for (int k = 0; k < km; k++) {
                if (G->solid[IDX(i, j, k)]) continue;
                const double t = S->t[IDX(i, j, k)];
                if (!(t > 0.0)) continue;
                const double b = P->g * S->p_stat[IDX(i, j, k)] / (P->r_mix * P->R_mix * t * P->t_ref);
                if (!isfinite(b)) continue;
                sum += wgt * b;
                wsum += wgt;
            }
        }
        S->buoy_ref[i] = (wsum > 0.0) ? sum / wsum : 0.0;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* RungeKutta_Jup_Turb.cpp:119-259. With ATJUP_METRIC_SPLIT (default) the column integral carries
 * (v^2 + w^2)/r + cor * w (plus the buoyancy only under ATJUP_HYDRO_SPLIT); otherwise the
 * buoyancy alone, integrated upward from the fluid foot of the column.                        */
static double buoy_term(const AtjupParams* P, const ora_state* S, size_t c, int i) {
    const double T = S->t[c];
    if (!(T > 0.0)) return 0.0;
    const double b = P->g * S->p_stat[c] / (P->r_mix * P->R_mix * T * P->t_ref) - S->buoy_ref[i];
    /* the ATJUP_BUOY_RHO_LEVEL form follows hydro_split; plain form otherwise */
    double f;
    if (P->hydro_split) {
        const double nd_rel = P->g * (P->L_atm * 1.0e3) / (P->u_0 * P->u_0);
        f = -nd_rel * P->buoy_scale * P->buoyancy * b / S->buoy_ref[i];
    } else {
        f = -P->nd_buoy * P->buoy_scale * P->buoyancy * b;
    }
    return isfinite(f) ? f : 0.0;
}

void ora_hydrostatic(const AtjupParams* P, const ora_grid* G, ora_state* S) {
    const int im = P->im, jm = P->jm, km = P->km;
    for (int j = 0; j < jm; j++) {
        const double cor = P->coriolis_split
            ? P->Coriolis * P->nd_cor * 2.0 * P->omega * fabs(sin(G->the[j])) : 0.0;
        for (int k = 0; k < km; k++) {
            int i0 = 0;
            while (i0 < im && G->solid[IDX(i0, j, k)]) { S->p_hydro[IDX(i0, j, k)] = 0.0; i0++; }
            if (i0 >= im) continue;
            int i1 = i0;
            while (i1 + 1 < im && !G->solid[IDX(i1 + 1, j, k)]) i1++;
            for (int i = i1 + 1; i < im; i++) S->p_hydro[IDX(i, j, k)] = 0.0;
            if (P->metric_split) {
                S->p_hydro[IDX(i0, j, k)] = 0.0;
                double fprev = 0.0;
                for (int i = i0; i <= i1; i++) {
                    const size_t c = IDX(i, j, k);
                    const double vv = S->v[c], ww = S->w[c];
                    const double f = (P->hydro_split ? buoy_term(P, S, c, i) : 0.0)
                                   + ((vv * vv + ww * ww) / G->rad[i] + cor * ww) / 1.0;
                    if (i > i0)
                        S->p_hydro[c] = S->p_hydro[IDX(i - 1, j, k)] + 0.5 * (fprev + f) * P->dr;
                    fprev = f;
                }
                if (S->p_baro)
                    for (int i = i0; i <= i1; i++) S->p_hydro[IDX(i, j, k)] += S->p_baro[IDX(i, j, k)];
            } else {
                S->p_hydro[IDX(i0, j, k)] = 0.0;
                for (int i = i0 + 1; i <= i1; i++)
                    S->p_hydro[IDX(i, j, k)] = S->p_hydro[IDX(i - 1, j, k)]
                        + 0.5 * (buoy_term(P, S, IDX(i - 1, j, k), i - 1) + buoy_term(P, S, IDX(i, j, k), i)) * P->dr;
            }
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* RHS_Jup_Turb.cpp:31-1457, the dynamics equations. Reads the live fields t, u, v, w (the
 * stage input), writes rhs_t/u/v/w and aux_u/v/w at (i, j, k).                               */
void ora_rhs_cell(const AtjupParams* P, const ora_grid* G, ora_state* S, int i, int j, int k) {
    const int im = P->im, jm = P->jm, km = P->km;
    (void)im;
    geom g;
    make_geom(P, G, i, j, &g);
    const int per = 1;
    const int kw = phi_wrap(per, k - 1, km), ke = phi_wrap(per, k + 1, km);
    const size_t c = IDX(i, j, k);
    const size_t cip = IDX(i + 1, j, k), cim = IDX(i - 1, j, k);
    const size_t cjp = IDX(i, j + 1, k), cjm = IDX(i, j - 1, k);
    const size_t ckp = IDX(i, j, ke), ckm = IDX(i, j, kw);
    const uint8_t* sol = G->solid;

    const double u_ijk = S->u[c], v_ijk = S->v[c], w_ijk = S->w[c];

    /* pgrad: centred difference with solid faces mirrored to the local value (103-130) */
#define PGRAD(Pf, hi_i, lo_i, inv2d) ( \
        ((P->pgrad_wall && sol[hi_i]) ? (Pf)[c] : (Pf)[hi_i]) - \
        ((P->pgrad_wall && sol[lo_i]) ? (Pf)[c] : (Pf)[lo_i])) * (inv2d)

#define DR1(F) ((F[cip] - F[cim]) * g.inv_2dr * g.exp_rm)
#define DR2(F) ((F[cip] - 2.0 * F[c] + F[cim]) * g.inv_dr2 * g.exp_2_rm)
#define DT1(F) ((F[cjp] - F[cjm]) * g.inv_2dthe)
#define DT2(F) ((F[cjp] - 2.0 * F[c] + F[cjm]) * g.inv_dthe2)
#define DP1(F) ((F[ckp] - F[ckm]) * g.inv_2dphi)
#define DP2(F) ((F[ckp] - 2.0 * F[c] + F[ckm]) * g.inv_dphi2)

    const double *U = S->u, *V = S->v, *W = S->w, *T = S->t;
    const double dudr = DR1(U), d2udr2 = DR2(U), dvdr = DR1(V), d2vdr2 = DR2(V);
    const double dwdr = DR1(W), d2wdr2 = DR2(W), dtdr = DR1(T), d2tdr2 = DR2(T);
    const double dpdr = PGRAD(S->p_dyn, cip, cim, g.inv_2dr) * g.exp_rm;
    const double dudthe = DT1(U), d2udthe2 = DT2(U), dvdthe = DT1(V), d2vdthe2 = DT2(V);
    const double dwdthe = DT1(W), d2wdthe2 = DT2(W), dtdthe = DT1(T), d2tdthe2 = DT2(T);
    const double dpdthe = PGRAD(S->p_dyn, cjp, cjm, g.inv_2dthe);
    const double dudphi = DP1(U), d2udphi2 = DP2(U), dvdphi = DP1(V), d2vdphi2 = DP2(V);
    const double dwdphi = DP1(W), d2wdphi2 = DP2(W), dtdphi = DP1(T), d2tdphi2 = DP2(T);
    const double dpdphi = PGRAD(S->p_dyn, ckp, ckm, g.inv_2dphi);

    /* body forces (334-423): true sine in Coriolis and centrifugal terms */
    const double sinthe_true = sqrt(dmax(0.0, 1.0 - g.costhe * g.costhe));
    const double Coriolis_rad = P->nd_cor * -2.0 * P->omega * sinthe_true * w_ijk;
    const double Coriolis_the = P->nd_cor * -2.0 * P->omega * g.costhe * w_ijk;
    double v_cor = v_ijk, u_cor = u_ijk;
    if (P->cell_hold && G->cell_vbar0) {
        v_cor -= G->cell_vbar0[(size_t)i * jm + j];
        u_cor -= G->cell_ubar0[(size_t)i * jm + j];
    }
    const double Coriolis_phi = P->nd_cor * +2.0 * P->omega * (+g.costhe * v_cor + sinthe_true * u_cor);
    const double centrifugal_rad = P->nd_cent * P->omega * P->omega * g.rm * sinthe_true * sinthe_true;
    const double centrifugal_the = P->nd_cent * P->omega * P->omega * g.rm * sinthe_true * g.costhe;
    const double coeff_energy_p = P->u_0 * P->u_0 / (P->cp_mix * P->t_ref);

    const double v_invrm = v_ijk * g.inv_rm;
    const double w_invrs = w_ijk * g.inv_rmsinthe;

    /* compression work with the hydrostatic part (459-482) */
    double dpstatdr = 0.0;
    if (P->adiabatic) {
        const double to_nd = 1.0 / P->p_dyn_to_bar;
        dpstatdr = (S->p_stat[cip] - S->p_stat[cim]) * g.inv_2dr * g.exp_rm * to_nd;
        const double rho_l = S->rho_mix[c];
        if (P->adiabatic_rho && rho_l > 0.0 && isfinite(rho_l)) dpstatdr *= P->r_mix / rho_l;
    }
    const double pressure_t = coeff_energy_p
        * (u_ijk * (dpdr + dpstatdr) + v_invrm * dpdthe + w_invrs * dpdphi);
    const double transport_t = u_ijk * dtdr + v_invrm * dtdthe + w_invrs * dtdphi;

    const double metric_on = P->metric_split ? 0.0 : 1.0;
    const double cor_rad_on = P->coriolis_split ? 0.0 : 1.0;
    const double transport_u = u_ijk * dudr + v_invrm * dudthe + w_invrs * dudphi
        - metric_on * (v_ijk * v_ijk + w_ijk * w_ijk) * g.inv_rm;
    const double transport_v = u_ijk * dvdr + v_invrm * dvdthe + w_invrs * dvdphi
        + (u_ijk * v_ijk - w_ijk * w_ijk * g.cotanthe) * g.inv_rm;
    const double transport_w = u_ijk * dwdr + v_invrm * dwdthe + w_invrs * dwdphi
        + (w_ijk * u_ijk + v_ijk * w_ijk * g.cotanthe) * g.inv_rm;

    /* diffusion (521-545) */
    const double two_inv_rm = 2.0 * g.inv_rm;
    const double v_metric = (1.0 + g.costhe / (g.sinthe2)) * g.inv_rm2;
    const double diffusion_t = d2tdr2 + dtdr * two_inv_rm + d2tdthe2 * g.inv_rm2
        + dtdthe * g.costhe_inv_rm2sinthe + d2tdphi2 * g.inv_rm2sinthe2;
    const double diffusion_u = d2udr2 + 2.0 * u_ijk * g.inv_rm2 + d2udthe2 * g.inv_rm2
        + 4.0 * dudr * g.inv_rm + dudthe * g.costhe_inv_rm2sinthe
        + d2udphi2 * g.inv_rm2sinthe2;
    const double diffusion_v = d2vdr2 + dvdr * two_inv_rm + d2vdthe2 * g.inv_rm2
        + dvdthe * g.costhe_inv_rm2sinthe - v_metric * v_ijk
        + d2vdphi2 * g.inv_rm2sinthe2
        + 2.0 * dudthe * g.inv_rm2
        - dwdphi * 2.0 * g.costhe * g.inv_rm2sinthe2;
    const double diffusion_w = d2wdr2 + dwdr * two_inv_rm + d2wdthe2 * g.inv_rm2
        + dwdthe * g.costhe_inv_rm2sinthe - v_metric * w_ijk
        + d2wdphi2 * g.inv_rm2sinthe2
        + 2.0 * dudphi * g.inv_rm2sinthe
        + dvdphi * 2.0 * g.costhe * g.inv_rm2sinthe2;

    /* pressure-gradient terms (589-620) */
    const double dpdr_term = P->pgrad_scale * dpdr;
    const double dpdthe_term = P->pgrad_scale * dpdthe * g.inv_rm;
    const double dpdphi_term = P->pgrad_scale * dpdphi * g.inv_rmsinthe;
    double dphdthe_term = 0.0, dphdphi_term = 0.0;
    if (P->hydro_split || P->metric_split) {
        dphdthe_term = PGRAD(S->p_hydro, cjp, cjm, g.inv_2dthe) * g.inv_rm;
        dphdphi_term = PGRAD(S->p_hydro, ckp, ckm, g.inv_2dphi) * g.inv_rmsinthe;
    }

    /* radiative and latent heating (646-718) */
    double radiation_t = 0.0, precip_t = 0.0;
    if (P->has_heating && S->Q_rad && P->rad_coupling != 0.0) {
        const double T_phys = S->t[c] * P->t_ref;
        const double P_phys = S->p_stat[c] * 1.0e5;
        const double rho_f = S->rho_mix[c];
        const double rho = (rho_f > 0.0 && isfinite(rho_f)) ? rho_f
                         : ((T_phys > 1.0) ? P_phys / (P->R_mix * T_phys) : 0.0);
        const double L_rad = P->L_atm * 1.0e3;
        if (rho > 0.0 && P->cp_mix > 0.0) {
            radiation_t = P->rad_coupling * S->Q_rad[c] * L_rad / (rho * P->cp_mix * P->u_0 * P->t_ref);
            if (!isfinite(radiation_t)) radiation_t = 0.0;
            else if (radiation_t > 0.5) radiation_t = 0.5;
            else if (radiation_t < -0.5) radiation_t = -0.5;
        }
    }
    if (P->has_heating && S->Q_precip && P->precip_coupling != 0.0) {
        const double L_rad = P->L_atm * 1.0e3;
        double rho_p = P->r_mix;
        if (P->precip_rho_local && P->local_rho) {
            const double rr = S->rho_mix[c];
            rho_p = (rr > 0.0 && isfinite(rr)) ? rr : P->r_mix;
        }
        if (rho_p > 0.0 && P->cp_mix > 0.0) {
            precip_t = P->precip_coupling * S->Q_precip[c] * L_rad / (rho_p * P->cp_mix * P->u_0 * P->t_ref);
            if (!isfinite(precip_t)) precip_t = 0.0;
            else if (precip_t > 0.5) precip_t = 0.5;
            else if (precip_t < -0.5) precip_t = -0.5;
        }
    }

    /* eddy and wall viscosity (736-752) */
    double nue_t = 0.0;
    if (P->has_nue && S->nue && P->turb_coupling != 0.0 && isfinite(S->nue[c]))
        nue_t = P->turb_coupling * dmax(0.0, S->nue[c]);
    const double nue_t_s = nue_t / 0.9;
    const double nue_wall = S->wall_nue[c];

    S->rhs_t[c] = +pressure_t - transport_t
        + diffusion_t * (P->t_diff_scale / (P->re * P->pr) + nue_t_s)
        + radiation_t + precip_t;

    /* Boussinesq buoyancy anomaly (1080-1092) */
    const double buoyancy_u = (S->t[c] > 0.0)
        ? -P->nd_buoy * P->buoy_scale * P->buoy_ramp * P->buoyancy
          * (P->g * S->p_stat[c] / (P->r_mix * P->R_mix * S->t[c] * P->t_ref) - S->buoy_ref[i])
        : 0.0;

    const double visc = 1.0 / P->re + nue_t + nue_wall;
    S->rhs_u[c] = -dpdr_term + ((P->hydro_split != 0) ? 0.0 : buoyancy_u) - transport_u
        + diffusion_u * visc - cor_rad_on * P->Coriolis * Coriolis_rad
        + P->centrifugal * centrifugal_rad;
    S->rhs_v[c] = -dpdthe_term - dphdthe_term - transport_v + diffusion_v * visc
        - P->Coriolis * Coriolis_the + P->centrifugal * centrifugal_the;
    S->rhs_w[c] = -dpdphi_term - dphdphi_term - transport_w + diffusion_w * visc
        - P->Coriolis * Coriolis_phi;

    S->aux_u[c] = S->rhs_u[c] + dpdr_term;
    S->aux_v[c] = S->rhs_v[c] + dpdthe_term;
    S->aux_w[c] = S->rhs_w[c] + dpdphi_term;
#undef PGRAD
#undef DR1
#undef DR2
#undef DT1
#undef DT2
#undef DP1
#undef DP2
}

/* ------------------------------------------------------------------------------------------ */
/* RungeKutta_Jup_Turb.cpp:261-583: level mean, hydrostatic pressure, four separated stages
 * (pass A: RHS everywhere from one consistent state; pass B: accumulate and form the next
 * stage input), final assembly y = y_n + dt (k1 + 2k2 + 2k3 + k4) / 6.                       */
void ora_rk4(const AtjupParams* P, const ora_grid* G, ora_state* S) {
    const int im = P->im, jm = P->jm, km = P->km;
    ora_buoy_ref_level(P, G, S);
    ora_hydrostatic(P, G, S);
    const double dt = P->dt;
    for (int stage = 0; stage < 4; stage++) {
        const double c_in = (stage == 0 || stage == 1) ? 0.5 * dt : (stage == 2 ? dt : 0.0);
        const double wgt = (stage == 0 || stage == 3) ? 1.0 : 2.0;
        #pragma omp parallel for schedule(static)
        for (int i = 1; i < im - 1; i++)
            for (int j = 3; j < jm - 3; j++)
                for (int k = 0; k < km - 1; k++) {
                    if (G->solid[IDX(i, j, k)]) continue;
                    ora_rhs_cell(P, G, S, i, j, k);
                }
        #pragma omp parallel for schedule(static)
        for (int i = 1; i < im - 1; i++)
            for (int j = 3; j < jm - 3; j++)
                for (int k = 0; k < km - 1; k++) {
                    const size_t c = IDX(i, j, k);
                    if (G->solid[c]) continue;
                    S->acc_t[c] = (stage == 0) ? wgt * S->rhs_t[c] : S->acc_t[c] + wgt * S->rhs_t[c];
                    S->acc_u[c] = (stage == 0) ? wgt * S->rhs_u[c] : S->acc_u[c] + wgt * S->rhs_u[c];
                    S->acc_v[c] = (stage == 0) ? wgt * S->rhs_v[c] : S->acc_v[c] + wgt * S->rhs_v[c];
                    S->acc_w[c] = (stage == 0) ? wgt * S->rhs_w[c] : S->acc_w[c] + wgt * S->rhs_w[c];
                    if (stage < 3) {
                        S->t[c] = S->tn[c] + c_in * S->rhs_t[c];
                        S->u[c] = S->un[c] + c_in * S->rhs_u[c];
                        S->v[c] = S->vn[c] + c_in * S->rhs_v[c];
                        S->w[c] = S->wn[c] + c_in * S->rhs_w[c];
                    }
                }
    }
    const double one_sixth = 1.0 / 6.0;
    #pragma omp parallel for schedule(static)
    for (int i = 1; i < im - 1; i++)
        for (int j = 3; j < jm - 3; j++)
            for (int k = 0; k < km - 1; k++) {
                const size_t c = IDX(i, j, k);
                if (G->solid[c]) continue;
                S->t[c] = S->tn[c] + dt * S->acc_t[c] * one_sixth;
                S->u[c] = S->un[c] + dt * S->acc_u[c] * one_sixth;
                S->v[c] = S->vn[c] + dt * S->acc_v[c] * one_sixth;
                S->w[c] = S->wn[c] + dt * S->acc_w[c] * one_sixth;
            }
}

/* ------------------------------------------------------------------------------------------ */
/* cJupiterModel.cpp:1842-1864: radial walls of the projection source before the divergence.   */
void ora_prepare_projection(const AtjupParams* P, const ora_grid* G, ora_state* S) {
    const int im = P->im, jm = P->jm, km = P->km;
    (void)G;
    for (int j = 1; j < jm - 1; j++)
        for (int k = 0; k < km - 1; k++) {
            if (P->rigid_lid) {
                S->aux_u[IDX(0, j, k)] = 0.0;
                S->aux_u[IDX(im - 1, j, k)] = 0.0;
            } else {
                S->aux_u[IDX(0, j, k)] = C43 * S->aux_u[IDX(1, j, k)] - C13 * S->aux_u[IDX(2, j, k)];
                S->aux_u[IDX(im - 1, j, k)] = C43 * S->aux_u[IDX(im - 2, j, k)] - C13 * S->aux_u[IDX(im - 3, j, k)];
            }
            S->aux_v[IDX(0, j, k)] = C43 * S->aux_v[IDX(1, j, k)] - C13 * S->aux_v[IDX(2, j, k)];
            S->aux_v[IDX(im - 1, j, k)] = C43 * S->aux_v[IDX(im - 2, j, k)] - C13 * S->aux_v[IDX(im - 3, j, k)];
            S->aux_w[IDX(0, j, k)] = C43 * S->aux_w[IDX(1, j, k)] - C13 * S->aux_w[IDX(2, j, k)];
            S->aux_w[IDX(im - 1, j, k)] = C43 * S->aux_w[IDX(im - 2, j, k)] - C13 * S->aux_w[IDX(im - 3, j, k)];
        }
}

/* ------------------------------------------------------------------------------------------ */
/* PressureSolver.h:144-766, pointwise branch. The divergence source of one cell (370-459),
 * one-sided at solid cells, then the clamp |src| <= cap * den (484-487).                      */
static double pressure_cell_source(const AtjupParams* P, const ora_grid* G, const ora_state* S,
                                   int i, int j, int k, double den, const geom* g) {
    const int im = P->im, jm = P->jm, km = P->km;
    const uint8_t* sol = G->solid;
    const int kw = phi_wrap(1, k - 1, km), ke = phi_wrap(1, k + 1, km);
    const double inv_dthe = 1.0 / P->dthe, inv_dphi = 1.0 / P->dphi;
    const double *Su = S->aux_u, *Sv = S->aux_v, *Sw = S->aux_w;
    const int sld = sol[IDX(i, j, k)];
    const int sld_kp1 = sol[IDX(i, j, ke)], sld_km1 = sol[IDX(i, j, kw)];
    const int sld_kp2 = (k < km - 2) ? sol[IDX(i, j, k + 2)] : 0;
    const int sld_km2 = (k > 2) ? sol[IDX(i, j, k - 2)] : 0;
    const int i_in_range = (i < im - 2);
    const int j_inner = (j > 2) && (j < jm - 2);
    double du_dr = 0.0, dv_dthe = 0.0, dw_dphi = 0.0;
    int r_flag = 0, the_flag = 0, phi_flag = 0;
    if (i_in_range && sld && !sol[IDX(i + 1, j, k)]) {
        du_dr = (-3.0 * Su[IDX(i, j, k)] + 4.0 * Su[IDX(i + 1, j, k)] - Su[IDX(i + 2, j, k)]) * g->inv_2dr;
        r_flag = 1;
    }
    if (j_inner) {
        const int air_jp1 = !sol[IDX(i, j + 1, k)], air_jm1 = !sol[IDX(i, j - 1, k)];
        if (sld && air_jp1 && !sol[IDX(i, j + 2, k)]) {
            dv_dthe = (-3.0 * Sv[IDX(i, j, k)] + 4.0 * Sv[IDX(i, j + 1, k)] - Sv[IDX(i, j + 2, k)]) * g->inv_2dthe;
            the_flag = 1;
        }
        if (sld && air_jm1 && !sol[IDX(i, j - 2, k)]) {
            dv_dthe = -(-3.0 * Sv[IDX(i, j, k)] + 4.0 * Sv[IDX(i, j - 1, k)] - Sv[IDX(i, j - 2, k)]) * g->inv_2dthe;
            the_flag = 1;
        }
        if ((sld && air_jp1 && sol[IDX(i, j + 2, k)]) || (j == jm - 2 && !sld && sol[IDX(i, j + 1, k)])) {
            dv_dthe = (Sv[IDX(i, j + 1, k)] - Sv[IDX(i, j, k)]) * inv_dthe;
            the_flag = 1;
        }
        if ((sld && air_jm1 && sol[IDX(i, j - 2, k)]) || (j == 1 && sld && air_jm1)) {
            dv_dthe = (Sv[IDX(i, j - 1, k)] - Sv[IDX(i, j, k)]) * inv_dthe;
            the_flag = 1;
        }
    }
    if (k > 2 && k < km - 2) {
        const int air_kp1 = !sld_kp1, air_km1 = !sld_km1;
        if (sld && air_kp1 && !sld_kp2) {
            dw_dphi = (-3.0 * Sw[IDX(i, j, k)] + 4.0 * Sw[IDX(i, j, k + 1)] - Sw[IDX(i, j, k + 2)]) * g->inv_2dphi;
            phi_flag = 1;
        }
        if (sld && air_km1 && !sld_km2) {
            dw_dphi = -(-3.0 * Sw[IDX(i, j, k)] + 4.0 * Sw[IDX(i, j, k - 1)] - Sw[IDX(i, j, k - 2)]) * g->inv_2dphi;
            phi_flag = 1;
        }
        if ((sld && air_kp1 && sld_kp2) || (k == km - 2 && !sld && sld_kp1)) {
            dw_dphi = (Sw[IDX(i, j, k + 1)] - Sw[IDX(i, j, k)]) * inv_dphi;
            phi_flag = 1;
        }
        if ((sld && air_km1 && sld_km2) || (k == 1 && sld && air_km1)) {
            dw_dphi = (Sw[IDX(i, j, k - 1)] - Sw[IDX(i, j, k)]) * inv_dphi;
            phi_flag = 1;
        }
    }
    if (!r_flag) du_dr = (Su[IDX(i + 1, j, k)] - Su[IDX(i - 1, j, k)]) * g->inv_2dr;
    if (!the_flag) dv_dthe = (Sv[IDX(i, j + 1, k)] - Sv[IDX(i, j - 1, k)]) * g->inv_2dthe;
    if (!phi_flag) dw_dphi = (Sw[IDX(i, j, ke)] - Sw[IDX(i, j, kw)]) * g->inv_2dphi;
    double div_src = du_dr * g->exp_rm + dv_dthe * g->inv_rm + dw_dphi * g->inv_rmsinthe;
    const double src_max = den * P->p_dyn_cap;
    if (!isfinite(div_src)) div_src = 0.0;
    else if (div_src > src_max) div_src = src_max;
    else if (div_src < -src_max) div_src = -src_max;
    return div_src;
}

/* Stencil weights of row (i, j) (PressureSolver.h:354-357) with the solver's sine table. */
static void press_weights(const AtjupParams* P, const ora_grid* G, int i, int j, geom* g,
                          double* num1, double* num2, double* num3) {
    make_geom(P, G, i, j, g);
    /* PressureSolver.h:156-162: the same floor; the sine is never 0 on this grid's interior */
    *num1 = g->exp_2_rm * g->inv_dr2;
    *num2 = g->inv_rm2 * g->inv_dthe2;
    *num3 = g->inv_rm2sinthe2 * g->inv_dphi2;
}

/* Face-dropping sum over the six neighbours (461-479); returns den, writes acc. */
static double press_gather(const AtjupParams* P, const ora_grid* G, const double* p,
                           int i, int j, int k, double num1, double num2, double num3,
                           double* acc_out) {
    const int jm = P->jm, km = P->km;
    const uint8_t* sol = G->solid;
    const int kw = phi_wrap(1, k - 1, km), ke = phi_wrap(1, k + 1, km);
    const int sld = sol[IDX(i, j, k)];
    double acc = 0.0, den;
    if (P->press_wall && !sld) {
        den = 0.0;
        if (!sol[IDX(i + 1, j, k)]) { acc += num1 * p[IDX(i + 1, j, k)]; den += num1; }
        if (!sol[IDX(i - 1, j, k)]) { acc += num1 * p[IDX(i - 1, j, k)]; den += num1; }
        if (!sol[IDX(i, j + 1, k)]) { acc += num2 * p[IDX(i, j + 1, k)]; den += num2; }
        if (!sol[IDX(i, j - 1, k)]) { acc += num2 * p[IDX(i, j - 1, k)]; den += num2; }
        if (!sol[IDX(i, j, ke)]) { acc += num3 * p[IDX(i, j, ke)]; den += num3; }
        if (!sol[IDX(i, j, kw)]) { acc += num3 * p[IDX(i, j, kw)]; den += num3; }
    } else {
        den = 2.0 * num1 + 2.0 * num2 + 2.0 * num3;
        acc = (p[IDX(i + 1, j, k)] + p[IDX(i - 1, j, k)]) * num1
            + (p[IDX(i, j + 1, k)] + p[IDX(i, j - 1, k)]) * num2
            + (p[IDX(i, j, ke)] + p[IDX(i, j, kw)]) * num3;
    }
    *acc_out = acc;
    return den;
}

/* Boundary folds after each sweep (718-746): 2-point Neumann in r, then theta, seam copy. */
static void press_fold(const AtjupParams* P, double* p) {
    const int im = P->im, jm = P->jm, km = P->km;
    for (int k = 0; k < km; k++)
        for (int j = 0; j < jm; j++) {
            p[IDX(0, j, k)] = C43 * p[IDX(1, j, k)] - C13 * p[IDX(2, j, k)];
            p[IDX(im - 1, j, k)] = C43 * p[IDX(im - 2, j, k)] - C13 * p[IDX(im - 3, j, k)];
        }
    for (int k = 0; k < km; k++)
        for (int i = 0; i < im; i++) {
            p[IDX(i, 0, k)] = C43 * p[IDX(i, 1, k)] - C13 * p[IDX(i, 2, k)];
            p[IDX(i, jm - 1, k)] = C43 * p[IDX(i, jm - 2, k)] - C13 * p[IDX(i, jm - 3, k)];
        }
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++) p[IDX(i, j, km - 1)] = p[IDX(i, j, 0)];
}

void ora_pressure_source(const AtjupParams* P, const ora_grid* G, ora_state* S, double* src) {
    const int im = P->im, jm = P->jm, km = P->km;
    memset(src, 0, sizeof(double) * (size_t)im * jm * km);
    for (int i = 1; i < im - 1; i++)
        for (int j = 1; j < jm - 1; j++) {
            geom g; double n1, n2, n3;
            press_weights(P, G, i, j, &g, &n1, &n2, &n3);
            for (int k = 0; k < km - 1; k++) {
                double acc;
                const double den = press_gather(P, G, S->p_dyn, i, j, k, n1, n2, n3, &acc);
                if (den <= 0.0) continue;
                src[IDX(i, j, k)] = pressure_cell_source(P, G, S, i, j, k, den, &g);
            }
        }
}

void ora_pressure_sweeps(const AtjupParams* P, const ora_grid* G, ora_state* S, int sweeps,
                         double omega, const double* b) {
    const int im = P->im, jm = P->jm, km = P->km;
    ora_prepare_projection(P, G, S);
    double* p = S->p_dyn;
    for (int sweep = 0; sweep < sweeps; sweep++) {
        for (int colour = 0; colour < 2; colour++) {
            for (int i = 1; i < im - 1; i++)
                for (int j = 1; j < jm - 1; j++) {
                    geom g; double n1, n2, n3;
                    press_weights(P, G, i, j, &g, &n1, &n2, &n3);
                    for (int k = 0; k < km - 1; k++) {
                        if (((i + j + k) & 1) != colour) continue;
                        double acc;
                        const double den = press_gather(P, G, p, i, j, k, n1, n2, n3, &acc);
                        if (den <= 0.0) continue;
                        const double src = b ? b[IDX(i, j, k)]
                                             : pressure_cell_source(P, G, S, i, j, k, den, &g);
                        const double pgs = (acc - src) / den;
                        p[IDX(i, j, k)] = (omega == 1.0) ? pgs
                                        : p[IDX(i, j, k)] + omega * (pgs - p[IDX(i, j, k)]);
                    }
                }
        }
        press_fold(P, p);
    }
}

/* A p = sum over kept faces of num (p_nb - p), with the boundary values read as the folds set
 * them from the interior (the fixed point of the sweep satisfies A p = src). Evaluated as a sum of
 * differences so that a large smooth p (the solution's column-constant part is ~1e6 times the
 * source) loses no digits to cancellation: a folded face contributes num (1/3)(p_c - p_in).   */
void ora_pressure_apply(const AtjupParams* P, const ora_grid* G, const double* p, double* Ap) {
    const int im = P->im, jm = P->jm, km = P->km;
    const size_t N = (size_t)im * jm * km;
    const uint8_t* sol = G->solid;
    memset(Ap, 0, sizeof(double) * N);
    for (int i = 1; i < im - 1; i++)
        for (int j = 1; j < jm - 1; j++) {
            geom g; double n1, n2, n3;
            press_weights(P, G, i, j, &g, &n1, &n2, &n3);
            for (int k = 0; k < km - 1; k++) {
                const size_t c = IDX(i, j, k);
                const int kw = phi_wrap(1, k - 1, km), ke = phi_wrap(1, k + 1, km);
                const double pc = p[c];
                double s = 0.0;
                if (!sol[c] || !P->press_wall) {
                    /* radial faces */
                    if (!sol[IDX(i + 1, j, k)] || !P->press_wall)
                        s += (i + 1 == im - 1) ? n1 * C13 * (pc - p[IDX(i - 1, j, k)]) : n1 * (p[IDX(i + 1, j, k)] - pc);
                    if (!sol[IDX(i - 1, j, k)] || !P->press_wall)
                        s += (i - 1 == 0) ? n1 * C13 * (pc - p[IDX(i + 1, j, k)]) : n1 * (p[IDX(i - 1, j, k)] - pc);
                    if (!sol[IDX(i, j + 1, k)] || !P->press_wall)
                        s += (j + 1 == jm - 1) ? n2 * C13 * (pc - p[IDX(i, j - 1, k)]) : n2 * (p[IDX(i, j + 1, k)] - pc);
                    if (!sol[IDX(i, j - 1, k)] || !P->press_wall)
                        s += (j - 1 == 0) ? n2 * C13 * (pc - p[IDX(i, j + 1, k)]) : n2 * (p[IDX(i, j - 1, k)] - pc);
                    if (!sol[IDX(i, j, ke)] || !P->press_wall) s += n3 * (p[IDX(i, j, ke)] - pc);
                    if (!sol[IDX(i, j, kw)] || !P->press_wall) s += n3 * (p[IDX(i, j, kw)] - pc);
                }
                Ap[c] = s;
            }
        }
}

/* ------------------------------------------------------------------------------------------ */
void ora_mixture_density(const AtjupParams* P, const ora_grid* G, ora_state* S) {
    const int im = P->im, jm = P->jm, km = P->km;
    (void)G;
    const double pdyn_w = P->rho_pdyn ? 1.0 : 0.0;
    const size_t N = (size_t)im * jm * km;
    for (size_t c = 0; c < N; c++) {
        const double T = S->t[c] * P->t_ref;
        if (!(T > 0.0)) { S->rho_mix[c] = 0.0; continue; }
        const double p_pa = (S->p_stat[c] + pdyn_w * S->p_dyn[c] * P->p_dyn_to_bar) * 1.0e5;
        const double rho = p_pa / (P->R_mix * T);
        S->rho_mix[c] = isfinite(rho) ? rho : 0.0;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* BC_Jup.h:185-263 wrapping BoundaryConditions.h:151-250 for the dynamics fields t, u, v, w:
 * zonal means of v, w at levels im-3, im-2 before the pass; 2-point Neumann at both radial
 * walls; rigid lid u = 0; the top taper, then the zonal-mean-preserving sponge (taper 3).     */
/* The field lists of the boundary passes (BC_Jup.h:275-350), restricted to the fields of the
 * hot path: the diagnostics of the chemistry and force routines (j_*, jT_*, w_*, difflux_*,
 * thermalmassflux, the force arrays, Q_Latent, Q_Sensible) and chrom (off by default) are not
 * part of it. X == NULL: the dynamics fields only. */
enum { BCL_RADIUS, BCL_THETA_X, BCL_THETA_Z, BCL_PHI, BCL_SOLID, BCL_SPECIES };
/* the diffusive chemistry fluxes are in the radius, theta-zero, phi and solid lists */
static int add_difflux(ora_phys* X, double** L, int n) {
    for (int q = 0; q < 3; q++)
        if (X->difflux[q]) L[n++] = X->difflux[q];
    return n;
}
static int bc_list(int which, ora_state* S, ora_phys* X, double** L) {
    int n = 0;
    switch (which) {
    case BCL_RADIUS:
        L[n++] = S->t; L[n++] = S->u; L[n++] = S->v; L[n++] = S->w;
        if (X) {
            for (int s = 0; s < ATJUP_S_COUNT; s++) L[n++] = X->q[s];
            L[n++] = (double*)X->massflux_h2s; L[n++] = (double*)X->massflux_nh3;
            L[n++] = (double*)X->massflux_nh4sh;
            L[n++] = X->tke; L[n++] = X->dis; L[n++] = X->nue_out; L[n++] = X->prod;
            L[n++] = X->tke_source; L[n++] = X->dis_source;
            n = add_difflux(X, L, n);
        }
        break;
    case BCL_THETA_X:
        L[n++] = S->t; L[n++] = S->u;
        if (X) {
            for (int s = 0; s < ATJUP_S_COUNT; s++) L[n++] = X->q[s];
            L[n++] = X->tke; L[n++] = X->dis; L[n++] = X->nue_out; L[n++] = X->prod;
            L[n++] = X->tke_source; L[n++] = X->dis_source;
        }
        break;
    case BCL_THETA_Z:
        L[n++] = S->v; L[n++] = S->w;
        if (X) {
            L[n++] = (double*)X->massflux_h2s; L[n++] = (double*)X->massflux_nh3;
            L[n++] = (double*)X->massflux_nh4sh; L[n++] = (double*)X->fluxlim_nh4sh;
            n = add_difflux(X, L, n);
        }
        break;
    case BCL_PHI:
        L[n++] = S->t; L[n++] = S->u; L[n++] = S->v; L[n++] = S->w;
        if (X) {
            for (int s = 0; s < ATJUP_S_COUNT; s++) L[n++] = X->q[s];
            L[n++] = (double*)X->massflux_h2s; L[n++] = (double*)X->massflux_nh3;
            L[n++] = (double*)X->massflux_nh4sh; L[n++] = (double*)X->fluxlim_nh4sh;
            L[n++] = X->tke; L[n++] = X->dis; L[n++] = X->nue_out; L[n++] = X->prod;
            L[n++] = X->tke_source; L[n++] = X->dis_source;
            n = add_difflux(X, L, n);
        }
        break;
    case BCL_SOLID:   /* t and p_stat first: they keep their value where nothing is extrapolated */
        L[n++] = S->t; L[n++] = S->p_stat; L[n++] = S->p_dyn;
        if (X) {
            for (int s = 0; s < ATJUP_S_COUNT; s++) L[n++] = X->q[s];
            L[n++] = (double*)X->massflux_h2s; L[n++] = (double*)X->massflux_nh3;
            L[n++] = (double*)X->massflux_nh4sh; L[n++] = (double*)X->fluxlim_nh4sh;
            n = add_difflux(X, L, n);
        }
        break;
    case BCL_SPECIES:
        if (X) for (int s = 0; s < ATJUP_S_COUNT; s++) L[n++] = X->q[s];
        break;
    }
    return n;
}

/* BC_Jup::bcRadius (BC_Jup.h:185-263) around BoundaryConditions::bcRadius (151-250): 2-point
 * Neumann at both radial walls for every listed field, rigid lid u = 0, the top taper of v, w
 * (3 = zonal-mean preserving), then the species wall copy at i = 0 and positivity at both walls. */
void ora_bc_radius_x(const AtjupParams* P, const ora_grid* G, ora_state* S, ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km, kn = km - 1;
    (void)G;
    double* zm = NULL;
    if (P->top_taper == 3) {
        zm = (double*)calloc((size_t)4 * jm, sizeof(double));
        for (int j = 0; j < jm; j++)
            for (int l = 0; l < 2; l++) {
                const int i = im - 3 + l;
                double sv = 0.0, sw = 0.0;
                for (int k = 0; k < kn; k++) { sv += S->v[IDX(i, j, k)]; sw += S->w[IDX(i, j, k)]; }
                zm[(size_t)(2 * l) * jm + j] = sv / kn;
                zm[(size_t)(2 * l + 1) * jm + j] = sw / kn;
            }
    }
    double* F[40];
    const int nf = bc_list(BCL_RADIUS, S, X, F);
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++)
            for (int f = 0; f < nf; f++) {
                F[f][IDX(0, j, k)] = C43 * F[f][IDX(1, j, k)] - C13 * F[f][IDX(2, j, k)];
                F[f][IDX(im - 1, j, k)] = C43 * F[f][IDX(im - 2, j, k)] - C13 * F[f][IDX(im - 3, j, k)];
            }
    if (P->lid_u)
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++) { S->u[IDX(0, j, k)] = 0.0; S->u[IDX(im - 1, j, k)] = 0.0; }
    if (P->top_taper != 0) {
        const int iml = im - 1;
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++) {
                S->v[IDX(iml, j, k)] = 0.0;
                S->w[IDX(iml, j, k)] = 0.0;
                if (P->top_taper == 2) {
                    S->v[IDX(iml - 1, j, k)] = (1.0 / 3.0) * S->v[IDX(iml - 3, j, k)];
                    S->w[IDX(iml - 1, j, k)] = (1.0 / 3.0) * S->w[IDX(iml - 3, j, k)];
                    S->v[IDX(iml - 2, j, k)] = (2.0 / 3.0) * S->v[IDX(iml - 3, j, k)];
                    S->w[IDX(iml - 2, j, k)] = (2.0 / 3.0) * S->w[IDX(iml - 3, j, k)];
                } else {
                    S->v[IDX(iml - 1, j, k)] *= (1.0 / 3.0);
                    S->w[IDX(iml - 1, j, k)] *= (1.0 / 3.0);
                    S->v[IDX(iml - 2, j, k)] *= (2.0 / 3.0);
                    S->w[IDX(iml - 2, j, k)] *= (2.0 / 3.0);
                }
            }
    }
    if (zm) {
        for (int j = 0; j < jm; j++) {
            const double v3 = zm[j], w3 = zm[(size_t)jm + j];
            const double v2 = zm[(size_t)2 * jm + j], w2 = zm[(size_t)3 * jm + j];
            for (int k = 0; k < km; k++) {
                S->v[IDX(im - 3, j, k)] += (1.0 / 3.0) * v3;
                S->w[IDX(im - 3, j, k)] += (1.0 / 3.0) * w3;
                S->v[IDX(im - 2, j, k)] += (2.0 / 3.0) * v2;
                S->w[IDX(im - 2, j, k)] += (2.0 / 3.0) * w2;
                S->v[IDX(im - 1, j, k)] = v2;
                S->w[IDX(im - 1, j, k)] = w2;
            }
        }
        free(zm);
    }
    /* species: wall copy (ATJUP_BC_SPECIES_WALL_COPY 1), positivity (ATJUP_BC_RADIUS_POSITIVE 1) */
    double* Q[ATJUP_S_COUNT];
    const int nq = bc_list(BCL_SPECIES, S, X, Q);
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++)
            for (int f = 0; f < nq; f++) Q[f][IDX(0, j, k)] = Q[f][IDX(1, j, k)];
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++)
            for (int f = 0; f < nq; f++) {
                if (Q[f][IDX(0, j, k)] < 0.0) Q[f][IDX(0, j, k)] = 0.0;
                if (Q[f][IDX(im - 1, j, k)] < 0.0) Q[f][IDX(im - 1, j, k)] = 0.0;
            }
}

/* BoundaryConditions.h:253-336: fill the rows next to the poles that the RK step does not
 * integrate (copy for the extrapolated list, ramp for the zero list), then the pole rows (copy;
 * zero list = 0).                                                                              */
void ora_bc_theta_x(const AtjupParams* P, const ora_grid* G, ora_state* S, ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    (void)G;
    const int nfill = P->pole_fill_rows;
    double *XL[40], *Z[40];
    const int nx = bc_list(BCL_THETA_X, S, X, XL), nz = bc_list(BCL_THETA_Z, S, X, Z);
    for (int k = 0; k < km; k++)
        for (int i = 0; i < im; i++) {
            if (nfill > 0) {
                const int jf = nfill + 1;
                for (int r = 1; r <= nfill; r++) {
                    const double ramp = (double)r / (double)jf;
                    for (int f = 0; f < nx; f++) {
                        XL[f][IDX(i, r, k)] = XL[f][IDX(i, jf, k)];
                        XL[f][IDX(i, jm - 1 - r, k)] = XL[f][IDX(i, jm - 1 - jf, k)];
                    }
                    for (int f = 0; f < nz; f++) {
                        Z[f][IDX(i, r, k)] = ramp * Z[f][IDX(i, jf, k)];
                        Z[f][IDX(i, jm - 1 - r, k)] = ramp * Z[f][IDX(i, jm - 1 - jf, k)];
                    }
                }
            }
            for (int f = 0; f < nz; f++) { Z[f][IDX(i, 0, k)] = 0.0; Z[f][IDX(i, jm - 1, k)] = 0.0; }
            for (int f = 0; f < nx; f++) {
                XL[f][IDX(i, 0, k)] = XL[f][IDX(i, 1, k)];             /* pole copy (form COPY) */
                XL[f][IDX(i, jm - 1, k)] = XL[f][IDX(i, jm - 2, k)];
            }
        }
}

/* BoundaryConditions.h:339-360: periodic seam, k = km-1 is the copy of k = 0. */
void ora_bc_phi_x(const AtjupParams* P, const ora_grid* G, ora_state* S, ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    (void)G;
    double* F[40];
    const int nf = bc_list(BCL_PHI, S, X, F);
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            for (int f = 0; f < nf; f++) F[f][IDX(i, j, km - 1)] = F[f][IDX(i, j, 0)];
}

/* BC_Jup.h:460-658: velocities 0 in solid cells; surface cells take the 2-point extrapolation
 * of every listed scalar from the first direction with two fluid cells (+i, -i, +j, -j, +k, -k),
 * interior cells (and surface cells without a pair) set the list from p_dyn on to 0; then solid
 * t = ambient row mean; then (with the physics fields) the sanitising clamps of k*, omega*, nue,
 * prod and the sources over the whole grid, n copies included. */
void ora_bc_solid_x(const AtjupParams* P, const ora_grid* G, ora_state* S, ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    const uint8_t* sol = G->solid;
#define SOLID(ii, jj, kk) (((ii) < 0 || (ii) >= im || (jj) < 0 || (jj) >= jm || (kk) < 0 || (kk) >= km) ? 1 : sol[IDX(ii, jj, kk)])
#define FLUID(ii, jj, kk) (((ii) < 0 || (ii) >= im || (jj) < 0 || (jj) >= jm || (kk) < 0 || (kk) >= km) ? 0 : !sol[IDX(ii, jj, kk)])
    double* sc[40];
    const int ns = bc_list(BCL_SOLID, S, X, sc);
    const int n_state = 2;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++)
            for (int i = 0; i < im; i++) {
                const size_t c = IDX(i, j, k);
                if (!sol[c]) continue;
                S->u[c] = 0.0; S->v[c] = 0.0; S->w[c] = 0.0;
                const int surf = !SOLID(i + 1, j, k) || !SOLID(i - 1, j, k) || !SOLID(i, j + 1, k)
                              || !SOLID(i, j - 1, k) || !SOLID(i, j, k + 1) || !SOLID(i, j, k - 1);
                if (!surf) { for (int f = n_state; f < ns; f++) sc[f][c] = 0.0; continue; }
                int ok = 1; size_t a = 0, b = 0;
                if (FLUID(i + 1, j, k) && FLUID(i + 2, j, k)) { a = IDX(i + 1, j, k); b = IDX(i + 2, j, k); }
                else if (FLUID(i - 1, j, k) && FLUID(i - 2, j, k)) { a = IDX(i - 1, j, k); b = IDX(i - 2, j, k); }
                else if (FLUID(i, j + 1, k) && FLUID(i, j + 2, k)) { a = IDX(i, j + 1, k); b = IDX(i, j + 2, k); }
                else if (FLUID(i, j - 1, k) && FLUID(i, j - 2, k)) { a = IDX(i, j - 1, k); b = IDX(i, j - 2, k); }
                else if (FLUID(i, j, k + 1) && FLUID(i, j, k + 2)) { a = IDX(i, j, k + 1); b = IDX(i, j, k + 2); }
                else if (FLUID(i, j, k - 1) && FLUID(i, j, k - 2)) { a = IDX(i, j, k - 1); b = IDX(i, j, k - 2); }
                else ok = 0;
                if (ok) { for (int f = 0; f < ns; f++) sc[f][c] = C43 * sc[f][a] - C13 * sc[f][b]; }
                else { for (int f = n_state; f < ns; f++) sc[f][c] = 0.0; }
            }
    if (P->mount_t_ambient)
        for (int i = 0; i < im; i++)
            for (int j = 0; j < jm; j++) {
                double s = 0.0; int n = 0, any = 0;
                for (int k = 0; k < km; k++) {
                    if (sol[IDX(i, j, k)]) { any = 1; continue; }
                    s += S->t[IDX(i, j, k)]; n++;
                }
                if (!any || n == 0) continue;
                const double t_amb = s / n;
                for (int k = 0; k < km; k++) if (sol[IDX(i, j, k)]) S->t[IDX(i, j, k)] = t_amb;
            }
    if (X) {
        const size_t N = (size_t)im * jm * km;
        const double tke_max_nd = 1000.0 / (P->u_0 * P->u_0);
        const double nue_max = 1.0e5 / (P->u_0 * P->L_atm * 1.0e3);
        const double prod_max = 1.0e4, dis_max = 1.0e6;
        for (size_t c = 0; c < N; c++) {
            X->tke[c] = safe_clamp(X->tke[c], 0.0, tke_max_nd);
            X->tken[c] = safe_clamp(X->tken[c], 0.0, tke_max_nd);
            X->dis[c] = safe_clamp(X->dis[c], 1.0e-10, dis_max);
            X->disn[c] = safe_clamp(X->disn[c], 1.0e-10, dis_max);
            X->nue_out[c] = safe_clamp(X->nue_out[c], 0.0, nue_max);
            X->prod[c] = safe_clamp(X->prod[c], 0.0, prod_max);
            X->tke_source[c] = safe_clamp(X->tke_source[c], -prod_max, prod_max);
            X->dis_source[c] = safe_clamp(X->dis_source[c], -prod_max, prod_max);
        }
    }
#undef SOLID
#undef FLUID
}

void ora_bc_radius(const AtjupParams* P, const ora_grid* G, ora_state* S) { ora_bc_radius_x(P, G, S, NULL); }
void ora_bc_theta(const AtjupParams* P, const ora_grid* G, ora_state* S) { ora_bc_theta_x(P, G, S, NULL); }
void ora_bc_phi(const AtjupParams* P, const ora_grid* G, ora_state* S) { ora_bc_phi_x(P, G, S, NULL); }
void ora_bc_solid(const AtjupParams* P, const ora_grid* G, ora_state* S) { ora_bc_solid_x(P, G, S, NULL); }

/* ------------------------------------------------------------------------------------------ */
/* lib/Utils.cpp:227-453. Direction-split k (periodic ring of km-1, seam copy), j (clamped),
 * i (clamped at the fluid floor); every pass reads a full copy of the field.                 */
void ora_shapiro(const AtjupParams* P, const ora_grid* G, double* f, int order, double strength,
                 int passes, int use_topo) {
    const int im = P->im, jm = P->jm, km = P->km;
    const size_t N = (size_t)im * jm * km;
    double* tmp = (double*)malloc(sizeof(double) * N);
    const double c4 = strength / 16.0, c2 = strength * 0.25;
#define TOPO(jj, kk) (use_topo ? (G->topo[(size_t)(jj) * km + (kk)] > 0 ? G->topo[(size_t)(jj) * km + (kk)] : 0) : 0)
#define INF(ii, jj, kk) ((ii) >= TOPO(jj, kk))
    for (int pass = 0; pass < passes; pass++) {
        /* k */
        memcpy(tmp, f, sizeof(double) * N);
        for (int i = 0; i < im; i++)
            for (int j = 0; j < jm; j++) {
                if (order == 4) {
                    const int n_k = km - 1;
                    for (int k = 0; k < n_k; k++) {
                        if (!INF(i, j, k)) continue;
                        const int km1 = (k - 1 + n_k) % n_k, kp1 = (k + 1) % n_k;
                        const int km2 = (k - 2 + n_k) % n_k, kp2 = (k + 2) % n_k;
                        const double cc = tmp[IDX(i, j, k)];
                        if (!INF(i, j, km1) || !INF(i, j, kp1)) continue;
                        if (INF(i, j, km2) && INF(i, j, kp2)) {
                            const double d4 = tmp[IDX(i, j, kp2)] - 4.0 * tmp[IDX(i, j, kp1)]
                                + 6.0 * cc - 4.0 * tmp[IDX(i, j, km1)] + tmp[IDX(i, j, km2)];
                            f[IDX(i, j, k)] = cc - c4 * d4;
                        } else {
                            f[IDX(i, j, k)] = cc + c2 * (tmp[IDX(i, j, km1)] - 2.0 * cc + tmp[IDX(i, j, kp1)]);
                        }
                    }
                } else {
                    for (int k = 0; k < km - 1; k++) {
                        if (!INF(i, j, k)) continue;
                        const int km1 = (k == 0) ? km - 2 : k - 1;
                        const int kp1 = (k == km - 2) ? 0 : k + 1;
                        const double v_km1 = INF(i, j, km1) ? tmp[IDX(i, j, km1)] : tmp[IDX(i, j, k)];
                        const double v_kp1 = INF(i, j, kp1) ? tmp[IDX(i, j, kp1)] : tmp[IDX(i, j, k)];
                        f[IDX(i, j, k)] = tmp[IDX(i, j, k)] + c2 * (v_km1 - 2.0 * tmp[IDX(i, j, k)] + v_kp1);
                    }
                }
                f[IDX(i, j, km - 1)] = f[IDX(i, j, 0)];
            }
        /* j */
        memcpy(tmp, f, sizeof(double) * N);
        for (int i = 0; i < im; i++)
            for (int j = 0; j < jm; j++)
                for (int k = 0; k < km; k++) {
                    if (!INF(i, j, k)) continue;
                    const double cc = tmp[IDX(i, j, k)];
                    if (order == 4) {
                        const int fm1 = (j - 1 >= 0) && INF(i, j - 1, k);
                        const int fp1 = (j + 1 <= jm - 1) && INF(i, j + 1, k);
                        if (!fm1 || !fp1) continue;
                        const int fm2 = (j - 2 >= 0) && INF(i, j - 2, k);
                        const int fp2 = (j + 2 <= jm - 1) && INF(i, j + 2, k);
                        if (fm2 && fp2) {
                            const double d4 = tmp[IDX(i, j + 2, k)] - 4.0 * tmp[IDX(i, j + 1, k)]
                                + 6.0 * cc - 4.0 * tmp[IDX(i, j - 1, k)] + tmp[IDX(i, j - 2, k)];
                            f[IDX(i, j, k)] = cc - c4 * d4;
                        } else {
                            f[IDX(i, j, k)] = cc + c2 * (tmp[IDX(i, j - 1, k)] - 2.0 * cc + tmp[IDX(i, j + 1, k)]);
                        }
                    } else {
                        const int jm1 = j - 1 > 0 ? j - 1 : 0, jp1 = j + 1 < jm - 1 ? j + 1 : jm - 1;
                        const double v_jm1 = INF(i, jm1, k) ? tmp[IDX(i, jm1, k)] : cc;
                        const double v_jp1 = INF(i, jp1, k) ? tmp[IDX(i, jp1, k)] : cc;
                        f[IDX(i, j, k)] = cc + c2 * (v_jm1 - 2.0 * cc + v_jp1);
                    }
                }
        /* i */
        memcpy(tmp, f, sizeof(double) * N);
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++) {
                const int i_surf = TOPO(j, k);
                for (int i = i_surf; i < im; i++) {
                    const double cc = tmp[IDX(i, j, k)];
                    if (order == 4) {
                        const int fm1 = (i - 1 >= i_surf), fp1 = (i + 1 <= im - 1);
                        if (!fm1 || !fp1) continue;
                        const int fm2 = (i - 2 >= i_surf), fp2 = (i + 2 <= im - 1);
                        if (fm2 && fp2) {
                            const double d4 = tmp[IDX(i + 2, j, k)] - 4.0 * tmp[IDX(i + 1, j, k)]
                                + 6.0 * cc - 4.0 * tmp[IDX(i - 1, j, k)] + tmp[IDX(i - 2, j, k)];
                            f[IDX(i, j, k)] = cc - c4 * d4;
                        } else {
                            f[IDX(i, j, k)] = cc + c2 * (tmp[IDX(i - 1, j, k)] - 2.0 * cc + tmp[IDX(i + 1, j, k)]);
                        }
                    } else {
                        const int im1 = i - 1 > i_surf ? i - 1 : i_surf, ip1 = i + 1 < im - 1 ? i + 1 : im - 1;
                        f[IDX(i, j, k)] = cc + c2 * (tmp[IDX(im1, j, k)] - 2.0 * cc + tmp[IDX(ip1, j, k)]);
                    }
                }
            }
    }
#undef TOPO
#undef INF
    free(tmp);
}

/* ------------------------------------------------------------------------------------------ */
/* InitValues_Jup.cpp:1500-1538: trapezoid column mean of r v over columns off the obstacle;
 * zonal form (default with ATJUP_VORTEX): per latitude the mean over meridians k < km-1 of the
 * column means is removed from every off-obstacle column of the row, all levels.              */
double ora_balance_column_v(const AtjupParams* P, const ora_grid* G, ora_state* S) {
    const int im = P->im, jm = P->jm, km = P->km;
    double vshift = 0.0;
    double* dvc = (double*)calloc((size_t)jm * km, sizeof(double));
    for (int j = 1; j < jm - 1; j++)
        for (int k = 0; k < km; k++) {
            const int i0 = G->topo[(size_t)j * km + k];
            if (i0 > 0) continue;
            double I1 = 0.0, I0 = 0.0;
            for (int i = i0; i < im - 1; i++) {
                I1 += 0.5 * (G->rad[i] * S->v[IDX(i, j, k)] + G->rad[i + 1] * S->v[IDX(i + 1, j, k)]) * P->dr;
                I0 += 0.5 * (G->rad[i] + G->rad[i + 1]) * P->dr;
            }
            const double dv = I1 / I0;
            if (P->v_massbal_zonal) { dvc[(size_t)j * km + k] = dv; continue; }
            for (int i = i0; i < im; i++) S->v[IDX(i, j, k)] -= dv;
            if (fabs(dv) > vshift) vshift = fabs(dv);
        }
    if (P->v_massbal_zonal)
        for (int j = 1; j < jm - 1; j++) {
            double s = 0.0; int n = 0;
            for (int k = 0; k < km - 1; k++)
                if (G->topo[(size_t)j * km + k] == 0) { s += dvc[(size_t)j * km + k]; n++; }
            if (!n) continue;
            const double dv = s / n;
            for (int k = 0; k < km; k++) {
                if (G->topo[(size_t)j * km + k] > 0) continue;
                for (int i = 0; i < im; i++) S->v[IDX(i, j, k)] -= dv;
            }
            if (fabs(dv) > vshift) vshift = fabs(dv);
        }
    free(dvc);
    return vshift;
}

/* ------------------------------------------------------------------------------------------ */
/* InitValues_Jup.cpp:1595-1822, projectAroundObstacle(in_loop = true): per level i = 1..im-2 that
 * cuts the obstacle, the box M = cone_proj_margin cells wider than the body's cross-section
 * (clipped to j 1..jm-2, k 1..km-2; phi = 0 one cell outside it), with H = cone_proj_div > 0 the
 * divergence solve (cells within H cells of the body, Chebyshev in 3-D, take s r D of the flow
 * before the correction as a source and close their wall faces), then the wall-flux solve; each
 * by lexicographic SOR (omega 1.9, stop at a largest change <= 1e-10 of the largest |phi|, at
 * most 40000 sweeps) from its phi of the previous call, then v, w incremented by the average of
 * the two face corrections (a wall face's correction is minus the cell's velocity); last the
 * seam copy of v and w. phi_div and phi_wall ([im*jm*km], zero before the first call) carry the
 * warm starts; sweeps (may be NULL) receives [2 * levels] sweep counts, the return value is the
 * number of levels.                                                                           */
static int cone_near(const AtjupParams* P, const ora_grid* G, int H, int i, int j, int k) {
    const int im = P->im, jm = P->jm, km = P->km;
    for (int di = -H; di <= H; di++) {
        const int ii = i + di;
        if (ii < 0 || ii >= im) continue;
        for (int dj = -H; dj <= H; dj++) {
            const int jj = j + dj;
            if (jj < 0 || jj >= jm) continue;
            for (int dk = -H; dk <= H; dk++) {
                const int kk = k + dk;
                if (kk < 0 || kk >= km) continue;
                if (G->solid[IDX(ii, jj, kk)]) return 1;
            }
        }
    }
    return 0;
}

int ora_cone_project(const AtjupParams* P, const ora_grid* G, ora_state* S, double* phi_div,
                     double* phi_wall, int32_t* sweeps) {
    const int im = P->im, jm = P->jm, km = P->km;
    const int H = P->cone_proj_div > 0 ? P->cone_proj_div : 0, M = P->cone_proj_margin;
    const double dr = P->dr, dthe = P->dthe, dphi = P->dphi, omega = 1.9;
    double* s = (double*)malloc(sizeof(double) * jm);
    for (int j = 0; j < jm; j++) {
        const double a = fabs(sin(G->the[j]));
        s[j] = a > P->sinthe_min ? a : P->sinthe_min;
    }
#define SOL(a, b, c) (G->solid[IDX(a, b, c)] != 0)
    int nlev = 0;
    for (int i = 1; i < im - 1; i++) {
        int jmin = jm, jmax = -1, kmin = km, kmax = -1;
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++)
                if (SOL(i, j, k)) {
                    if (j < jmin) jmin = j;
                    if (j > jmax) jmax = j;
                    if (k < kmin) kmin = k;
                    if (k > kmax) kmax = k;
                }
        if (jmax < 0) continue;
        const int jlo = jmin - M > 1 ? jmin - M : 1, jhi = jmax + M < jm - 2 ? jmax + M : jm - 2;
        const int klo = kmin - M > 1 ? kmin - M : 1, khi = kmax + M < km - 2 ? kmax + M : km - 2;
        if (jhi < jlo || khi < klo) continue;
        const int NJ = jhi - jlo + 1, NK = khi - klo + 1;
        uint8_t* nr = (uint8_t*)calloc((size_t)NJ * NK, 1);
        double* Gs = (double*)calloc((size_t)NJ * NK, sizeof(double));
        if (H > 0)
            for (int j = jlo; j <= jhi; j++)
                for (int k = klo; k <= khi; k++) {
                    if (SOL(i, j, k) || !cone_near(P, G, H, i, j, k)) continue;
                    nr[(size_t)(j - jlo) * NK + (k - klo)] = 1;
                    /* s r D, the 3-D face divergence with the wall faces closed (1653-1664) */
                    const double r = G->rad[i], rp = r + 0.5 * dr, rm = r - 0.5 * dr;
                    const double sj = s[j], sp = 0.5 * (sj + s[j + 1]), sm = 0.5 * (sj + s[j - 1]);
                    const double up = SOL(i + 1, j, k) ? 0.0 : 0.5 * (S->u[IDX(i, j, k)] + S->u[IDX(i + 1, j, k)]);
                    const double um = SOL(i - 1, j, k) ? 0.0 : 0.5 * (S->u[IDX(i, j, k)] + S->u[IDX(i - 1, j, k)]);
                    const double vp = SOL(i, j + 1, k) ? 0.0 : 0.5 * (S->v[IDX(i, j, k)] + S->v[IDX(i, j + 1, k)]);
                    const double vm = SOL(i, j - 1, k) ? 0.0 : 0.5 * (S->v[IDX(i, j, k)] + S->v[IDX(i, j - 1, k)]);
                    const double wp = SOL(i, j, k + 1) ? 0.0 : 0.5 * (S->w[IDX(i, j, k)] + S->w[IDX(i, j, k + 1)]);
                    const double wm = SOL(i, j, k - 1) ? 0.0 : 0.5 * (S->w[IDX(i, j, k)] + S->w[IDX(i, j, k - 1)]);
                    Gs[(size_t)(j - jlo) * NK + (k - klo)] =
                        sj * r * (rp * rp * up - rm * rm * um) / (r * r * dr) +
                        (sp * vp - sm * vm) / dthe + (wp - wm) / dphi;
                }
        for (int pass = H > 0 ? 0 : 1; pass < 2; pass++) {
            const int div = pass == 0;
            double* phi = div ? phi_div : phi_wall;     /* the box's phi lives at its cells */
            int it;
            for (it = 1; it <= 40000; it++) {
                double dmax = 0.0, pmax = 0.0;
                for (int j = jlo; j <= jhi; j++) {
                    const double aN = 0.5 * (s[j] + s[j - 1]) / (dthe * dthe);
                    const double aS = 0.5 * (s[j] + s[j + 1]) / (dthe * dthe);
                    const double aL = 1.0 / (s[j] * dphi * dphi);
                    for (int k = klo; k <= khi; k++) {
                        if (SOL(i, j, k)) continue;
                        /* phi of a neighbour outside the box is the halo's 0 */
                        const double pN = j - 1 >= jlo ? phi[IDX(i, j - 1, k)] : 0.0;
                        const double pS = j + 1 <= jhi ? phi[IDX(i, j + 1, k)] : 0.0;
                        const double pW = k - 1 >= klo ? phi[IDX(i, j, k - 1)] : 0.0;
                        const double pE = k + 1 <= khi ? phi[IDX(i, j, k + 1)] : 0.0;
                        const double vp = S->v[IDX(i, j, k)], wp = S->w[IDX(i, j, k)];
                        double A = 0.0, B = 0.0;
                        if (div && nr[(size_t)(j - jlo) * NK + (k - klo)]) {
                            if (!SOL(i, j - 1, k)) { A += aN; B += aN * pN; }
                            if (!SOL(i, j + 1, k)) { A += aS; B += aS * pS; }
                            if (!SOL(i, j, k - 1)) { A += aL; B += aL * pW; }
                            if (!SOL(i, j, k + 1)) { A += aL; B += aL * pE; }
                            B += Gs[(size_t)(j - jlo) * NK + (k - klo)];
                        } else {
                            if (SOL(i, j - 1, k)) B -= aN * dthe * (-vp); else { A += aN; B += aN * pN; }
                            if (SOL(i, j + 1, k)) B -= aS * dthe * (vp); else { A += aS; B += aS * pS; }
                            if (SOL(i, j, k - 1)) B -= aL * s[j] * dphi * (-wp); else { A += aL; B += aL * pW; }
                            if (SOL(i, j, k + 1)) B -= aL * s[j] * dphi * (wp); else { A += aL; B += aL * pE; }
                        }
                        if (!(A > 0.0)) continue;
                        double* pp = &phi[IDX(i, j, k)];
                        const double pn = *pp + omega * (B / A - *pp);
                        const double d = fabs(pn - *pp);
                        if (d > dmax) dmax = d;
                        *pp = pn;
                        if (fabs(pn) > pmax) pmax = fabs(pn);
                    }
                }
                if (dmax <= 1.0e-10 * (pmax > 1.0e-30 ? pmax : 1.0e-30)) break;
            }
            if (sweeps) sweeps[2 * nlev + pass] = it;
            for (int j = jlo; j <= jhi; j++)
                for (int k = klo; k <= khi; k++) {
                    if (SOL(i, j, k)) continue;
                    const double vp = S->v[IDX(i, j, k)], wp = S->w[IDX(i, j, k)];
                    const double pp = phi[IDX(i, j, k)];
                    const double pN = j - 1 >= jlo ? phi[IDX(i, j - 1, k)] : 0.0;
                    const double pS = j + 1 <= jhi ? phi[IDX(i, j + 1, k)] : 0.0;
                    const double pW = k - 1 >= klo ? phi[IDX(i, j, k - 1)] : 0.0;
                    const double pE = k + 1 <= khi ? phi[IDX(i, j, k + 1)] : 0.0;
                    const double dN = SOL(i, j - 1, k) ? -vp : (pp - pN) / dthe;
                    const double dS = SOL(i, j + 1, k) ? -vp : (pS - pp) / dthe;
                    const double dW = SOL(i, j, k - 1) ? -wp : (pp - pW) / (s[j] * dphi);
                    const double dE = SOL(i, j, k + 1) ? -wp : (pE - pp) / (s[j] * dphi);
                    S->v[IDX(i, j, k)] = vp + 0.5 * (dN + dS);
                    S->w[IDX(i, j, k)] = wp + 0.5 * (dW + dE);
                }
        }
        if (sweeps && H == 0) sweeps[2 * nlev] = 0;
        free(nr);
        free(Gs);
        nlev++;
    }
#undef SOL
    /* the seam copy (1806-1807) */
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++) {
            S->v[IDX(i, j, km - 1)] = S->v[IDX(i, j, 0)];
            S->w[IDX(i, j, km - 1)] = S->w[IDX(i, j, 0)];
        }
    free(s);
    return nlev;
}

void ora_restore(const AtjupParams* P, ora_state* S) {
    const size_t N = (size_t)P->im * P->jm * P->km;
    memcpy(S->tn, S->t, sizeof(double) * N);
    memcpy(S->un, S->u, sizeof(double) * N);
    memcpy(S->vn, S->v, sizeof(double) * N);
    memcpy(S->wn, S->w, sizeof(double) * N);
}

/* cJupiterModel.cpp:1032-1381 with the saturation adjustment, chemistry, radiation,
 * precipitation, turbulence, convective adjustment and cone projection off (dry config). */
void ora_iteration_dry(const AtjupParams* P, const ora_grid* G, ora_state* S, int iter_n,
                       int first, int sweeps) {
    if (iter_n % 2 == 0 || first) {
        ora_pressure_sweeps(P, G, S, sweeps, 1.0, NULL);
        ora_mixture_density(P, G, S);
    }
    ora_rk4(P, G, S);
    ora_bc_radius(P, G, S);
    ora_bc_theta(P, G, S);
    ora_bc_phi(P, G, S);
    ora_bc_solid(P, G, S);
    if (P->shapiro_inloop > 0) {
        ora_shapiro(P, G, S->u, 4, P->shapiro_strength, P->shapiro_inloop, 1);
        ora_shapiro(P, G, S->v, 4, P->shapiro_strength, P->shapiro_inloop, 1);
        ora_shapiro(P, G, S->w, 4, P->shapiro_strength, P->shapiro_inloop, 1);
    }
    if (P->v_massbal_stride > 0 && iter_n % P->v_massbal_stride == 0)
        ora_balance_column_v(P, G, S);
    ora_restore(P, S);
}

/* Size of the parameter block as compiled here, for binding checks. */
size_t ora_params_sizeof(void) { return sizeof(AtjupParams); }
size_t ora_micro_sizeof(void) { return sizeof(AtjupMicro); }
size_t ora_gas_params_sizeof(void) { return sizeof(AtjupGasParams); }
size_t ora_sat_stats_sizeof(void) { return sizeof(AtjupSatStats); }

/* ---------------------------------------------------------------------------------------------
 * Saturation adjustment of one gas (SaturationAdjustment.h:255-746; Tao, Simpson and McCumber
 * 1988). Every expression keeps the reference's operand order, so with the same libm this is
 * bit-identical to it. Print-only parts (budget sums, DIAG counters, the reported cell) are
 * left out; counts[0..2] = cells that entered the iteration, that used every pass, that left
 * through the dry exit.
 * ------------------------------------------------------------------------------------------- */

/* ATPhys.h:49-52: Clausius-Clapeyron fit [bar]; R in J/(kg K), coefficients per J/(g K). */
static double ora_svp(double T, double C, double L0, double R, double da, double db) {
    return exp(C + (-L0 / T + da * log(T) + db * T) / (1e-3 * R));
}

enum { SAT_PASSES = 15 };                 /* iter_prec_end, SaturationAdjustment.h:250 */
static const double SAT_Q_DIFF_MIN = 1.0e-3;  /* q_diff_min, SaturationAdjustment.h:251 */

/* Vapour target of a cell holding q_c liquid and q_i ice at temperature T, given the liquid and
 * ice saturation densities (SaturationAdjustment.h:513-520 and the same choice at 564-571). */
static double sat_target(const AtjupGasParams* g, double T, double q_c, double q_i, double q_l,
                         double q_s, double t_range_inv) {
    if (q_c > 0.0 && q_i > 0.0) return (q_c * q_l + q_i * q_s) / (q_c + q_i);
    if (g->bergeron >= 2 && q_c <= 0.0 && q_i <= 0.0 && T < g->t_0) return q_s;
    if (g->ice_entry && q_c <= 0.0 && q_i <= 0.0) {
        const double cn = T <= g->t_00 ? 0.0 : (T >= g->t_0 ? 1.0 : (T - g->t_00) * t_range_inv);
        return cn * q_l + (1.0 - cn) * q_s;
    }
    if (q_i == 0.0) return q_l;
    return q_s;
}

void ora_satadj(const AtjupParams* P, const ora_grid* G, const AtjupGasParams* g, double* t,
                const double* p_stat, const double* rho_mix, double* c, double* cloud,
                double* ice, long long* counts) {
    const int im = P->im, jm = P->jm, km = P->km;
    const size_t N = (size_t)im * jm * km;
    const double t_range_inv = 1.0 / (g->t_0 - g->t_00);
    const int freeze_on = g->freeze && g->conserve && g->t_00 > 0.0 && g->t_00 < g->t_0;
    const double Lf = g->ls - g->lv;
    const double cp = P->cp_mix;
    long long n_adj = 0, n_nc = 0, n_dry = 0;

    for (size_t q = 0; q < N; q++) {
        double t_u = t[q] * P->t_ref;
        const double p_u = p_stat[q];
        if (!(t_u > 0.0) || !(p_u > 0.0) || G->solid[q]) continue;
        /* rho_at (cJupiterModel.h:1212-1216) */
        double rho = P->r_mix;
        if (P->local_rho && rho_mix[q] > 0.0 && isfinite(rho_mix[q])) rho = rho_mix[q];

        /* entry bounds (SaturationAdjustment.h:368-407) */
        if (t_u > g->t_0) {
            if (g->conserve) {
                if (ice[q] > 0.0) {
                    double dm = ice[q];
                    if (Lf > 0.0) {
                        const double hc = cp * rho;
                        const double cap = hc * (t_u - g->t_0) / Lf;
                        if (dm > cap) dm = cap;
                        t_u -= Lf * dm / hc;
                        t[q] = t_u / P->t_ref;
                    }
                    ice[q] -= dm;
                    cloud[q] += dm;
                }
            } else {
                ice[q] = 0.0;
            }
        }
        if (freeze_on && t_u < g->t_00 && cloud[q] > 0.0) {
            double dm = cloud[q];
            if (Lf > 0.0) {
                const double hc = cp * rho;
                const double cap = hc * (g->t_00 - t_u) / Lf;
                if (dm > cap) dm = cap;
                t_u += Lf * dm / hc;
                t[q] = t_u / P->t_ref;
            }
            cloud[q] -= dm;
            ice[q] += dm;
        }
        if (c[q] < 0.0) c[q] = 0.0;
        if (cloud[q] < 0.0) cloud[q] = 0.0;
        if (ice[q] < 0.0) ice[q] = 0.0;

        /* entry test (SaturationAdjustment.h:422-452) */
        const double rho_c = rho;
        const double q_rain0 = rho_c * g->ep * ora_svp(t_u, g->C, g->L0, g->R, g->del_alf,
                                                        g->del_bet) / p_u;
        if (q_rain0 <= 0.0) continue;
        double q_entry = q_rain0;
        if (g->ice_entry && cloud[q] <= 0.0 && ice[q] <= 0.0) {
            const double cnd0 = t_u <= g->t_00 ? 0.0
                              : (t_u >= g->t_0 ? 1.0 : (t_u - g->t_00) * t_range_inv);
            if (cnd0 < 1.0)
                q_entry = cnd0 * q_rain0 + (1.0 - cnd0) * rho_c * g->ep
                        * ora_svp(t_u, g->C_i, g->L0_i, g->R, g->del_alf_i, g->del_bet_i) / p_u;
        }
        if (g->bergeron >= 2 && cloud[q] <= 0.0 && ice[q] <= 0.0 && t_u < g->t_0)
            q_entry = rho_c * g->ep * ora_svp(t_u, g->C_i, g->L0_i, g->R, g->del_alf_i,
                                              g->del_bet_i) / p_u;
        if (c[q] <= q_entry) {
            const double qc0 = cloud[q], qi0 = ice[q];
            if (!g->evap || !g->conserve || (qc0 <= 0.0 && qi0 <= 0.0)) continue;
            const double q_ice0 = rho_c * g->ep * ora_svp(t_u, g->C_i, g->L0_i, g->R,
                                                          g->del_alf_i, g->del_bet_i) / p_u;
            double q_t0;
            if (qc0 > 0.0 && qi0 > 0.0) q_t0 = (qc0 * q_rain0 + qi0 * q_ice0) / (qc0 + qi0);
            else if (qi0 <= 0.0) q_t0 = q_rain0;
            else q_t0 = q_ice0;
            if (fabs(c[q] - q_t0) <= SAT_Q_DIFF_MIN * q_t0) continue;
        }

        /* mixed-phase iteration (SaturationAdjustment.h:454-604) */
        double qv = c[q], qc = cloud[q], qi = ice[q], T = t_u, hyp = qv;
        double q_rain_now = q_rain0;
        int found = 0, dry = 0;
        const double heat = cp * rho_c;
        for (int itr = 1; itr <= SAT_PASSES; itr++) {
            double CND = (T - g->t_00) * t_range_inv;
            double DEP = (g->t_0 - T) * t_range_inv;
            if (T <= g->t_00) { CND = 0.0; DEP = 1.0; }
            if (T >= g->t_0) { CND = 1.0; DEP = 0.0; }
            const int berg = g->bergeron != 0 && T < g->t_0 && qv <= q_rain_now
                          && (qi > 0.0 || (g->bergeron >= 2 && qc <= 0.0));
            if (berg) {
                CND = 0.0; DEP = 1.0;
                if (qc > 0.0) {
                    T -= g->lv * qc / heat;
                    qv += qc;
                    qc = 0.0;
                }
            }
            double dv = hyp - qv;
            double dc = -dv * CND;
            double di = -dv * DEP;
            if (g->conserve) {
                if (dv < -qv) { dv = -qv; dc = -dv * CND; di = -dv * DEP; }
                if (qc + dc < 0.0) { const double ex = -(qc + dc); dc = -qc; di -= ex; }
                if (qi + di < 0.0) {
                    const double ex = -(qi + di); di = -qi; dc -= ex;
                    if (qc + dc < 0.0) dc = -qc;
                }
                dv = -(dc + di);
            }
            T += (g->lv * dc + g->ls * di) / heat;
            qv += dv;
            qc += dc;
            qi += di;
            if (qv < 0.0) qv = 0.0;
            if (qc < 0.0) qc = 0.0;
            if (qi < 0.0) qi = 0.0;

            const double q_l = rho_c * g->ep * ora_svp(T, g->C, g->L0, g->R, g->del_alf,
                                                       g->del_bet) / p_u;
            const double q_s = rho_c * g->ep * ora_svp(T, g->C_i, g->L0_i, g->R, g->del_alf_i,
                                                       g->del_bet_i) / p_u;
            q_rain_now = q_l;
            hyp = sat_target(g, T, qc, qi, q_l, q_s, t_range_inv);

            if (T >= g->t_0) {
                if (g->conserve) {
                    if (qi > 0.0) {
                        double dm = qi;
                        if (Lf > 0.0) {
                            const double cap = heat * (T - g->t_0) / Lf;
                            if (dm > cap) dm = cap;
                            T -= Lf * dm / heat;
                        }
                        qi -= dm;
                        qc += dm;
                    }
                } else {
                    qi = 0.0;
                }
            }
            const double q_diff = fabs(qv - hyp) / (hyp + 1e-20);
            if (q_diff <= SAT_Q_DIFF_MIN) { found = 1; break; }
            if (g->dry_exit && g->conserve && qc <= 0.0 && qi <= 0.0 && qv < hyp) { dry = 1; break; }
            if (g->newton) {
                const double dT = 0.1;
                const double q_ld = rho_c * g->ep * ora_svp(T + dT, g->C, g->L0, g->R,
                                                            g->del_alf, g->del_bet) / p_u;
                const double q_sd = rho_c * g->ep * ora_svp(T + dT, g->C_i, g->L0_i, g->R,
                                                            g->del_alf_i, g->del_bet_i) / p_u;
                const double hyp_d = sat_target(g, T, qc, qi, q_ld, q_sd, t_range_inv);
                double CNDn = (T - g->t_00) * t_range_inv;
                if (T <= g->t_00) CNDn = 0.0;
                if (T >= g->t_0) CNDn = 1.0;
                if (berg) CNDn = 0.0;
                const double G2 = (g->lv * CNDn + g->ls * (1.0 - CNDn)) / heat
                                * (hyp_d - hyp) / dT;
                double wgt = 1.0 / (1.0 + dmax(G2, 0.0));
                if (wgt < 0.05) wgt = 0.05;
                hyp = qv + wgt * (hyp - qv);
            } else {
                hyp = 0.5 * (hyp + qv);
            }
        }
        n_adj++;
        if (!found && !dry) n_nc++;
        if (dry) n_dry++;
        c[q] = qv;
        cloud[q] = qc;
        ice[q] = qi;
        t[q] = T / P->t_ref;
    }
    /* final clamp (SaturationAdjustment.h:673-685) */
    for (size_t q = 0; q < N; q++) {
        if (c[q] <= 0.0) c[q] = 0.0;
        if (cloud[q] <= 0.0) cloud[q] = 0.0;
        if (ice[q] <= 0.0) ice[q] = 0.0;
    }
    if (counts) { counts[0] = n_adj; counts[1] = n_nc; counts[2] = n_dry; }
}

/* ---------------------------------------------------------------------------------------------
 * Full physics in the RK4 step: the 11 species and k*, omega* (RHS_Jup_Turb.cpp:132-303 for the
 * derivatives, 482-545 transport and diffusion, 736-998 the closure sources, 1266-1452 the
 * right-hand sides; RungeKutta_Jup_Turb.cpp:419-568 the stage and final updates).
 * ------------------------------------------------------------------------------------------- */

/* m_layer_heights is float [km]; get_layer_height(i) is -1 outside 0..im-1 (cJupiterModel.h:
 * 133-138), layer_thickness_m(i) -1 outside 0..im-2 and the float difference times 1e3. */
static double layer_h(const ora_phys* X, int im, int i) {
    if (i < 0 || i > im - 1) return (double)(-1.0f);
    return (double)X->layer_heights[i];
}
static double layer_dz_m(const ora_phys* X, int im, int i) {
    if (i < 0 || i > im - 2) return -1.0;
    return (double)(X->layer_heights[i + 1] - X->layer_heights[i]) * 1.0e3;
}

/* Per-species diffusion Schmidt number and source terms (RHS_Jup_Turb.cpp:1273-1340). */
static double species_sc(const AtjupPhysics* PH, int s) {
    switch (s) {
    case ATJUP_S_H2O: case ATJUP_S_H2O_CLOUD: case ATJUP_S_H2O_ICE: return PH->sc_h2o;
    case ATJUP_S_H2S: return PH->sc_h2s;
    case ATJUP_S_NH3: case ATJUP_S_NH3_CLOUD: case ATJUP_S_NH3_ICE: return PH->sc_nh3;
    case ATJUP_S_CH4: case ATJUP_S_CH4_CLOUD: case ATJUP_S_CH4_ICE: return PH->sc_ch4;
    default: return PH->sc_nh4sh;
    }
}

/* index of the species' S_precip field in ora_phys.s_precip (-1: none) */
static int species_precip(int s) {
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

/* Right-hand sides of the species and of k*, omega* at one cell, from the live fields. */
void ora_rhs_phys_cell(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G,
                       ora_state* S, ora_phys* X, int i, int j, int k) {
    const int im = P->im, jm = P->jm, km = P->km;
    geom g;
    make_geom(P, G, i, j, &g);
    const int kw = phi_wrap(1, k - 1, km), ke = phi_wrap(1, k + 1, km);
    const size_t c = IDX(i, j, k);
    const size_t cip = IDX(i + 1, j, k), cim = IDX(i - 1, j, k);
    const size_t cjp = IDX(i, j + 1, k), cjm = IDX(i, j - 1, k);
    const size_t ckp = IDX(i, j, ke), ckm = IDX(i, j, kw);
    const double u_ijk = S->u[c], v_ijk = S->v[c], w_ijk = S->w[c];
    const double v_invrm = v_ijk * g.inv_rm;
    const double w_invrs = w_ijk * g.inv_rmsinthe;
    const double two_inv_rm = 2.0 * g.inv_rm;

    double nue_t = 0.0;
    if (P->has_nue && S->nue && P->turb_coupling != 0.0 && isfinite(S->nue[c]))
        nue_t = P->turb_coupling * dmax(0.0, S->nue[c]);
    const double nue_t_s = nue_t / 0.9;

#define DR1(F) ((F[cip] - F[cim]) * g.inv_2dr * g.exp_rm)
#define DR2(F) ((F[cip] - 2.0 * F[c] + F[cim]) * g.inv_dr2 * g.exp_2_rm)
#define DT1(F) ((F[cjp] - F[cjm]) * g.inv_2dthe)
#define DT2(F) ((F[cjp] - 2.0 * F[c] + F[cjm]) * g.inv_dthe2)
#define DP1(F) ((F[ckp] - F[ckm]) * g.inv_2dphi)
#define DP2(F) ((F[ckp] - 2.0 * F[c] + F[ckm]) * g.inv_dphi2)

    if (PH->species_on) {
        const double v_stokes = (2.0 / 9.0) * PH->r_p_nh4sh * PH->r_p_nh4sh
                              * (PH->rg_nh4sh - S->rho_mix[c]) * P->g / PH->mue_mix;
        for (int s = 0; s < ATJUP_S_COUNT; s++) {
            const double* F = X->q[s];
            const double d1r = DR1(F), d2r = DR2(F), d1t = DT1(F), d2t = DT2(F);
            const double d1p = DP1(F), d2p = DP2(F);
            const double transport = u_ijk * d1r + v_invrm * d1t + w_invrs * d1p;
            const double diffusion = d2r + d1r * two_inv_rm + d2t * g.inv_rm2
                + d1t * g.costhe_inv_rm2sinthe + d2p * g.inv_rm2sinthe2;
            const double coef = PH->species_diff_scale / (species_sc(PH, s) * P->re) + nue_t_s;
            const int ip = species_precip(s);
            double r;
            if (s == ATJUP_S_H2S) {
                r = -transport + diffusion * coef + PH->chemical_reaction * X->massflux_h2s[c];
            } else if (s == ATJUP_S_NH3) {
                r = -transport + diffusion * coef + PH->chemical_reaction * X->massflux_nh3[c]
                  + P->precip_coupling * X->s_precip[ip][c];
            } else if (s == ATJUP_S_NH4SH) {
                r = -transport + X->fluxlim_nh4sh[c] + diffusion * coef
                  + PH->chemical_reaction * X->massflux_nh4sh[c] + (v_stokes / P->u_0) * d1r;
            } else {
                r = -transport + diffusion * coef + P->precip_coupling * X->s_precip[ip][c];
            }
            X->rhs_q[s][c] = r;
        }
    }

    if (!PH->turb_on) {
        X->rhs_tke[c] = 0.0;
        X->rhs_dis[c] = 0.0;
        return;
    }
    /* derivatives of k*, omega*: central, solid neighbours replaced by the cell (257-303) */
    const double *TK = X->tke, *DS = X->dis;
    const uint8_t* sol = G->solid;
    double dtkedr = DR1(TK), d2tkedr2 = DR2(TK), ddisdr = DR1(DS), d2disdr2 = DR2(DS);
    double dtkedthe = DT1(TK), d2tkedthe2 = DT2(TK), ddisdthe = DT1(DS), d2disdthe2 = DT2(DS);
    double dtkedphi = DP1(TK), d2tkedphi2 = DP2(TK), ddisdphi = DP1(DS), d2disdphi2 = DP2(DS);
    {
        const int s_im = sol[cim], s_ip = sol[cip], s_jm = sol[cjm], s_jp = sol[cjp];
        const int s_km = sol[ckm], s_kp = sol[ckp];
        if (s_im || s_ip) {
            const double tm = s_im ? TK[c] : TK[cim], tp = s_ip ? TK[c] : TK[cip];
            const double dm = s_im ? DS[c] : DS[cim], dp = s_ip ? DS[c] : DS[cip];
            dtkedr = (tp - tm) * g.inv_2dr * g.exp_rm;
            d2tkedr2 = (tp - 2.0 * TK[c] + tm) * g.inv_dr2 * g.exp_2_rm;
            ddisdr = (dp - dm) * g.inv_2dr * g.exp_rm;
            d2disdr2 = (dp - 2.0 * DS[c] + dm) * g.inv_dr2 * g.exp_2_rm;
        }
        if (s_jm || s_jp) {
            const double tm = s_jm ? TK[c] : TK[cjm], tp = s_jp ? TK[c] : TK[cjp];
            const double dm = s_jm ? DS[c] : DS[cjm], dp = s_jp ? DS[c] : DS[cjp];
            dtkedthe = (tp - tm) * g.inv_2dthe;
            d2tkedthe2 = (tp - 2.0 * TK[c] + tm) * g.inv_dthe2;
            ddisdthe = (dp - dm) * g.inv_2dthe;
            d2disdthe2 = (dp - 2.0 * DS[c] + dm) * g.inv_dthe2;
        }
        if (s_km || s_kp) {
            const double tm = s_km ? TK[c] : TK[ckm], tp = s_kp ? TK[c] : TK[ckp];
            const double dm = s_km ? DS[c] : DS[ckm], dp = s_kp ? DS[c] : DS[ckp];
            dtkedphi = (tp - tm) * g.inv_2dphi;
            d2tkedphi2 = (tp - 2.0 * TK[c] + tm) * g.inv_dphi2;
            ddisdphi = (dp - dm) * g.inv_2dphi;
            d2disdphi2 = (dp - 2.0 * DS[c] + dm) * g.inv_dphi2;
        }
    }
    const double *U = S->u, *V = S->v, *W = S->w;
    const double dudr = DR1(U), dvdr = DR1(V), dwdr = DR1(W);
    const double dudthe = DT1(U), dvdthe = DT1(V), dwdthe = DT1(W);
    const double dudphi = DP1(U), dvdphi = DP1(V), dwdphi = DP1(W);
#undef DR1
#undef DR2
#undef DT1
#undef DT2
#undef DP1
#undef DP2
    const double transport_tke = u_ijk * dtkedr + v_invrm * dtkedthe + w_invrs * dtkedphi;
    const double transport_dis = u_ijk * ddisdr + v_invrm * ddisdthe + w_invrs * ddisdphi;
    const double diffusion_tke = d2tkedr2 + dtkedr * two_inv_rm + d2tkedthe2 * g.inv_rm2
        + dtkedthe * g.costhe_inv_rm2sinthe + d2tkedphi2 * g.inv_rm2sinthe2;
    const double diffusion_dis = d2disdr2 + ddisdr * two_inv_rm + d2disdthe2 * g.inv_rm2
        + ddisdthe * g.costhe_inv_rm2sinthe + d2disdphi2 * g.inv_rm2sinthe2;

    /* closure sources (781-998) */
    const double C_nue = 0.028, dis_min = 1.0e-10, nue_gas_phys = 1.8e-5;
    const double L_m = P->L_atm * 1.0e3;
    const double nue_max = PH->nue_max_phys / (P->u_0 * L_m);
    const double nue_here = (S->nue && isfinite(S->nue[c])) ? dmax(0.0, S->nue[c]) : 0.0;
    const double tke_c = TK[c], dis_c = DS[c];
    const double tke_s = dmax(tke_c, dis_min);
    const double dis_s = dmax(dis_c, dis_min);
    const double dudr_s = dudr, dvdr_s = dvdr, dwdr_s = dwdr;
    const double dudthe_s = dudthe * g.inv_rm, dvdthe_s = dvdthe * g.inv_rm;
    const double dwdthe_s = dwdthe * g.inv_rm;
    const double dudphi_s = dudphi * g.inv_rmsinthe, dvdphi_s = dvdphi * g.inv_rmsinthe;
    const double dwdphi_s = dwdphi * g.inv_rmsinthe;
    const double dtkedthe_s = dtkedthe * g.inv_rm, ddisdthe_s = ddisdthe * g.inv_rm;
    const double dtkedphi_s = dtkedphi * g.inv_rmsinthe, ddisdphi_s = ddisdphi * g.inv_rmsinthe;
    const double grad_dot = dtkedr * ddisdr + dtkedthe_s * ddisdthe_s + dtkedphi_s * ddisdphi_s;
    double cnue = (PH->turb_model == ATJUP_TURB_K_EPSILON) ? C_nue * tke_s * tke_s / dis_s
                                                           : tke_s / dis_s;
    cnue = dmin(cnue, nue_max);
    const double der = 0.66667 * (dudr_s + dvdthe_s + dwdphi_s);
    const double P_full = dmax(0.0,
          (cnue * (2.0 * dudr_s - der) - 0.66667 * tke_c) * dudr_s
        + (cnue * (dudthe_s + dvdr_s)) * dudthe_s
        + (cnue * (dudphi_s + dwdr_s)) * dudphi_s
        + (cnue * (2.0 * dvdthe_s - der) - 0.66667 * tke_c) * dvdthe_s
        + (cnue * (dvdr_s + dudthe_s)) * dvdr_s
        + (cnue * (dvdphi_s + dwdthe_s)) * dvdphi_s
        + (cnue * (2.0 * dwdphi_s - der) - 0.66667 * tke_c) * dwdphi_s
        + (cnue * (dwdr_s + dudphi_s)) * dwdr_s
        + (cnue * (dwdthe_s + dvdphi_s)) * dwdthe_s);
    X->prod[c] = P_full;

    const double y_mount = layer_h(X, im, G->topo[(size_t)j * km + k]) * 1.0e3;
    const double dz_layer = dmax(1.0, layer_dz_m(X, im, i - 1 > 0 ? i - 1 : 0));
    const double y_phys = dmax(layer_h(X, im, i) * 1.0e3 - y_mount, dz_layer);
    const double y_star = y_phys / L_m;

    double diffusion_tke_re = 0.0, diffusion_dis_re = 0.0, tke_src = 0.0, dis_src = 0.0;
    double c_w_prod = 0.0;
    if (PH->turb_model == ATJUP_TURB_K_EPSILON) {           /* Chien 1982 (799-829) */
        const double sig_k = 1.0, sig_w = 1.3, C_eps_1 = 1.35, C_eps_2 = 1.80;
        diffusion_tke_re = 1.0 / P->re + nue_here / sig_k;
        diffusion_dis_re = 1.0 / P->re + nue_here / sig_w;
        const double d_plus = y_phys * X->vel_star[(size_t)j * km + k] / nue_gas_phys;
        const double Re_T = tke_s * tke_s * P->u_0 * L_m / (dis_s * nue_gas_phys);
        const double f_2 = 1.0 - 0.4 / 1.8 * exp(-Re_T * Re_T / 36.0);
        const double y_star2 = y_star * y_star;
        const double L_k = -2.0 * tke_c / y_star2;
        const double L_w = -2.0 * dis_c / y_star2 * exp(-0.5 * d_plus);
        const double P_k = P_full;
        const double Y_k = dis_c;
        const double P_w = C_eps_1 * dis_c / tke_s * P_k;
        const double Y_w = C_eps_2 * f_2 * dis_c * dis_c / tke_s;
        tke_src = P_k - Y_k + L_k / PH->re_turb;
        dis_src = P_w - Y_w + L_w / PH->re_turb;
        c_w_prod = C_eps_1;
    } else if (PH->turb_model == ATJUP_TURB_K_OMEGA) {       /* Wilcox (830-875) */
        const double sig_k = 0.6, sig_w = 0.5, bet_star = 0.09, gam = 0.52, bet_0 = 0.0708;
        diffusion_tke_re = 1.0 / P->re + sig_k * nue_here;
        diffusion_dis_re = 1.0 / P->re + sig_w * nue_here;
        const double S11 = dudr_s, S22 = dvdthe_s, S33 = dwdphi_s;
        const double S12 = 0.5 * (dudthe_s + dvdr_s);
        const double S13 = 0.5 * (dudphi_s + dwdr_s);
        const double S23 = 0.5 * (dvdphi_s + dwdthe_s);
        const double S_mag = sqrt(2.0 * (S11 * S11 + S22 * S22 + S33 * S33
                                         + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23)));
        const double W12 = dudthe_s - dvdr_s;
        const double W13 = dudphi_s - dwdr_s;
        const double W23 = dvdphi_s - dwdthe_s;
        const double Omega = sqrt(W12 * W12 + W13 * W13 + W23 * W23);
        const double chi_w = fabs(Omega * Omega * S_mag / pow(bet_star * dis_s, 3));
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
    } else {                                                  /* SST, Menter 1994 (876-960) */
        const double bet_star = 0.09, sig_k1 = 1.176, sig_k2 = 1.0, sig_w1 = 2.0, sig_w2 = 1.168;
        const double bet1 = 0.0333, bet2 = 0.0368, gam1 = 0.413, gam2 = 0.2;
        const double nue_air_nd = nue_gas_phys / (P->u_0 * L_m);
        const double CD_kw = dmax(2.0 * sig_w2 / dis_s * grad_dot, 1.0e-20);
        const double arg1 = dmin(
            dmax(sqrt(dmax(tke_c, 0.0)) / (bet_star * dis_s * y_star),
                 500.0 * nue_air_nd / (y_star * y_star * dis_s)),
            4.0 * sig_w2 * tke_s / (CD_kw * y_star * y_star));
        const double F1 = tanh(pow(arg1, 4));
        const double sig_k = F1 * sig_k1 + (1.0 - F1) * sig_k2;
        const double sig_w = F1 * sig_w1 + (1.0 - F1) * sig_w2;
        diffusion_tke_re = 1.0 / P->re + nue_here / sig_k;
        diffusion_dis_re = 1.0 / P->re + nue_here / sig_w;
        const double P_k = dmin(P_full, 20.0 * bet_star * tke_s * dis_s);
        const double Y_k = bet_star * tke_s * dis_s;
        const double P_w = (F1 * gam1 + (1.0 - F1) * gam2) * P_k * dis_s / tke_s;
        const double Y_w = (F1 * bet1 + (1.0 - F1) * bet2) * dis_s * dis_s;
        const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_s * grad_dot;
        tke_src = P_k - Y_k;
        dis_src = P_w - Y_w + D_w;
        c_w_prod = F1 * gam1 + (1.0 - F1) * gam2;
    }
    if (PH->turb_buoy) {                                      /* ATJUP_TURB_BUOY (963-981) */
        const int ip = (i + 1 < im - 1) ? i + 1 : im - 1, imn = (i - 1 > 0) ? i - 1 : 0;
        const double dz_m = (layer_h(X, im, ip) - layer_h(X, im, imn)) * 1.0e3;
        const double T_K = dmax(S->t[c] * P->t_ref, 1.0);
        const double dTdz = (S->t[IDX(ip, j, k)] - S->t[IDX(imn, j, k)]) * P->t_ref / dmax(dz_m, 1.0);
        const double N2 = P->g / T_K * (dTdz + P->g / P->cp_mix);
        const double tscale = L_m / P->u_0;
        const double G_b = -(cnue / PH->turb_buoy_prt) * N2 * tscale * tscale;
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
    X->tke_source[c] = tke_src;
    X->dis_source[c] = dis_src;
    X->rhs_tke[c] = -transport_tke + diffusion_tke * diffusion_tke_re + tke_src;
    X->rhs_dis[c] = -transport_dis + diffusion_dis * diffusion_dis_re + dis_src;
}


/* RungeKutta_Jup_Turb.cpp:261-583 with every transported field. */
void ora_rk4_phys(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G, ora_state* S,
                  ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    ora_buoy_ref_level(P, G, S);
    ora_hydrostatic(P, G, S);
    const double dt = P->dt;
    const double tke_max_nd = PH->tke_max_phys / (P->u_0 * P->u_0);
    const double dis_min_nd = 1.0e-10;
    for (int stage = 0; stage < 4; stage++) {
        const double c_in = (stage == 0 || stage == 1) ? 0.5 * dt : (stage == 2 ? dt : 0.0);
        const double wgt = (stage == 0 || stage == 3) ? 1.0 : 2.0;
        /* each cell writes only its own right-hand sides and reads no other cell's: the loops
         * run in parallel with the same result to the bit */
        #pragma omp parallel for schedule(static)
        for (int i = 1; i < im - 1; i++)
            for (int j = 3; j < jm - 3; j++)
                for (int k = 0; k < km - 1; k++) {
                    if (G->solid[IDX(i, j, k)]) continue;
                    ora_rhs_cell(P, G, S, i, j, k);
                    ora_rhs_phys_cell(P, PH, G, S, X, i, j, k);
                }
        #pragma omp parallel for schedule(static)
        for (int i = 1; i < im - 1; i++)
            for (int j = 3; j < jm - 3; j++)
                for (int k = 0; k < km - 1; k++) {
                    const size_t c = IDX(i, j, k);
                    if (G->solid[c]) continue;
                    S->acc_t[c] = (stage == 0) ? wgt * S->rhs_t[c] : S->acc_t[c] + wgt * S->rhs_t[c];
                    S->acc_u[c] = (stage == 0) ? wgt * S->rhs_u[c] : S->acc_u[c] + wgt * S->rhs_u[c];
                    S->acc_v[c] = (stage == 0) ? wgt * S->rhs_v[c] : S->acc_v[c] + wgt * S->rhs_v[c];
                    S->acc_w[c] = (stage == 0) ? wgt * S->rhs_w[c] : S->acc_w[c] + wgt * S->rhs_w[c];
                    for (int s = 0; s < ATJUP_S_COUNT; s++)
                        X->acc_q[s][c] = (stage == 0) ? wgt * X->rhs_q[s][c]
                                                      : X->acc_q[s][c] + wgt * X->rhs_q[s][c];
                    X->acc_tke[c] = (stage == 0) ? wgt * X->rhs_tke[c] : X->acc_tke[c] + wgt * X->rhs_tke[c];
                    X->acc_dis[c] = (stage == 0) ? wgt * X->rhs_dis[c] : X->acc_dis[c] + wgt * X->rhs_dis[c];
                    if (stage < 3) {
                        S->t[c] = S->tn[c] + c_in * S->rhs_t[c];
                        S->u[c] = S->un[c] + c_in * S->rhs_u[c];
                        S->v[c] = S->vn[c] + c_in * S->rhs_v[c];
                        S->w[c] = S->wn[c] + c_in * S->rhs_w[c];
                        for (int s = 0; s < ATJUP_S_COUNT; s++)
                            X->q[s][c] = X->qn[s][c] + c_in * X->rhs_q[s][c];
                        X->tke[c] = safe_clamp(X->tken[c] + c_in * X->rhs_tke[c], 0.0, tke_max_nd);
                        X->dis[c] = dmax(dis_min_nd, X->disn[c] + c_in * X->rhs_dis[c]);
                    }
                }
    }
    const double one_sixth = 1.0 / 6.0;
    #pragma omp parallel for schedule(static)
    for (int i = 1; i < im - 1; i++)
        for (int j = 3; j < jm - 3; j++)
            for (int k = 0; k < km - 1; k++) {
                const size_t c = IDX(i, j, k);
                if (G->solid[c]) continue;
                S->t[c] = S->tn[c] + dt * S->acc_t[c] * one_sixth;
                S->u[c] = S->un[c] + dt * S->acc_u[c] * one_sixth;
                S->v[c] = S->vn[c] + dt * S->acc_v[c] * one_sixth;
                S->w[c] = S->wn[c] + dt * S->acc_w[c] * one_sixth;
                for (int s = 0; s < ATJUP_S_COUNT; s++) {
                    const double q = X->qn[s][c] + dt * X->acc_q[s][c] * one_sixth;
                    /* std::max(0.0, q), except NH4SH's explicit `if (q < 0) q = 0` (547-549),
                     * which keeps a NaN and a -0 */
                    X->q[s][c] = (s == ATJUP_S_NH4SH) ? (q < 0.0 ? 0.0 : q) : dmax(0.0, q);
                }
                X->tke[c] = safe_clamp(X->tken[c] + dt * X->acc_tke[c] * one_sixth, 0.0, tke_max_nd);
                X->dis[c] = dmax(dis_min_nd, X->disn[c] + dt * X->acc_dis[c] * one_sixth);
            }
}

/* Turbulence.h:383-422 apply_wall_bc: the wall law at the surface cell of obstacle columns, or
 * (ATJUP_TURB_FREE) row 0 copied from row 1. */
void ora_turb_wall_bc(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G, ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    const double C_nue = 0.028, nue_air = 1.8e-5;
    const double L_m = P->L_atm * 1.0e3;
    const int model = PH->turb_model;
    double *TK = X->tke, *DS = X->dis;
    const double nd_omega = L_m / P->u_0;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            const int i_w = G->topo[(size_t)j * km + k];
            if (!PH->turb_free && i_w > 0 && i_w < im - 1) {
                const double y1 = dmax(layer_dz_m(X, im, i_w - 1 > 0 ? i_w - 1 : 0), 1.0);
                const double vs = X->vel_star[(size_t)j * km + k];
                const size_t cw = IDX(i_w, j, k);
                TK[cw] = vs * vs / (sqrt(C_nue) * P->u_0 * P->u_0);
                X->nue_out[cw] = 0.0;
                if (model == ATJUP_TURB_K_EPSILON) DS[cw] = 0.0;
                else if (model == ATJUP_TURB_K_OMEGA) DS[cw] = 6.0 * nue_air / (0.075 * y1 * y1) * nd_omega;
                else DS[cw] = 60.0 * nue_air / (0.0333 * y1 * y1) * nd_omega;
            } else {
                TK[IDX(0, j, k)] = TK[IDX(1, j, k)];
                DS[IDX(0, j, k)] = DS[IDX(1, j, k)];
                X->nue_out[IDX(0, j, k)] = X->nue_out[IDX(1, j, k)];
            }
        }
}

/* turbWallOmega (cJupiterModel.cpp:360-377): omega* at the surface cell of obstacle columns
 * from the viscous and log-layer values. */
void ora_turb_wall_omega(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G, ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    if (!(PH->turb_wall_omega != 0 && PH->turb_model != ATJUP_TURB_K_EPSILON)) return;
    const double nue_air = 1.8e-5, bet_star = 0.09, bet_1 = 0.0333, kappa = 0.41;
    const double nd_omega = P->L_atm * 1.0e3 / P->u_0;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            const int i_w = G->topo[(size_t)j * km + k];
            if (i_w <= 0 || i_w >= im - 1) continue;
            const double y1 = dmax(layer_dz_m(X, im, i_w - 1 > 0 ? i_w - 1 : 0), 1.0);
            const double y = 0.5 * y1;
            const double om_vis = 60.0 * nue_air / (bet_1 * y1 * y1);
            const double om_log = X->vel_star[(size_t)j * km + k] / (sqrt(bet_star) * kappa * y);
            X->dis[IDX(i_w, j, k)] = sqrt(om_vis * om_vis + om_log * om_log) * nd_omega;
        }
}

/* ---------------------------------------------------------------------------------------------
 * The closure update between steps: Turbulence<cJupiterModel>::run (Turbulence.h:307-328) --
 * compute_vel_star (336-360), compute_sources with the separate clamp passes (614-882) and the
 * model routines (886-1106), apply_wall_bc (383-422), zero_land_cells (592-610), clamp_nue
 * (565-588), seam_copy (543-559), fill_lid_corners (511-536) -- then the driver's turbWallOmega
 * (cJupiterModel.cpp:360-377). ATJUP_TURB_CLAMP_PASS = 1 (the default) only.
 * ------------------------------------------------------------------------------------------- */
static double clamp3(double x, double lo, double hi) { return (x < lo) ? lo : ((x > hi) ? hi : x); }

void ora_turbulence(const AtjupParams* P, const AtjupPhysics* PH, const ora_grid* G, ora_state* S,
                    ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    const size_t N = (size_t)im * jm * km;
    const uint8_t* sol = G->solid;
    const double C_nue = 0.028, dis_min = 1.0e-10, nue_air = 1.8e-5;
    const double L_m = P->L_atm * 1.0e3;
    const double nue_max = PH->nue_max_phys / (P->u_0 * L_m);
    const int model = PH->turb_model;
    const double *U = S->u, *V = S->v, *W = S->w;
    double *TK = X->tke, *DS = X->dis;
#define HM(i_) (layer_h(X, im, (i_)) * 1.0e3)   /* height_m (Turbulence.h:263-265) */

    /* compute_vel_star */
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            double* vs = &X->vel_star[(size_t)j * km + k];
            if (PH->turb_free) { *vs = 0.05; continue; }
            int is = G->topo[(size_t)j * km + k] + 1;
            if (is > im - 1) is = im - 1;
            const double v_s = V[IDX(is, j, k)], w_s = W[IDX(is, j, k)];
            const double vw2 = v_s * v_s + w_s * w_s;
            if (!isfinite(vw2)) { *vs = 0.05; continue; }
            const double U_h = P->u_0 * sqrt(vw2);
            *vs = clamp3(sqrt(0.002) * U_h, 0.05, PH->vel_star_max);
        }

    /* compute_sources: clamp-in pass */
    for (int j = 1; j < jm - 1; j++)
        for (int k = 0; k < km - 1; k++)
            for (int i = 1; i < im - 1; i++) {
                const size_t c = IDX(i, j, k);
                if (sol[c]) continue;
                TK[c] = dmax(0.0, TK[c]);
                DS[c] = dmax(dis_min, DS[c]);
            }
    /* sources per cell */
    for (int j = 1; j < jm - 1; j++)
        for (int k = 0; k < km - 1; k++) {
            const int kw = phi_wrap(1, k - 1, km), ke = phi_wrap(1, k + 1, km);
            const double y_mount = HM(G->topo[(size_t)j * km + k]);
            for (int i = 1; i < im - 1; i++) {
                const size_t c = IDX(i, j, k);
                if (sol[c]) continue;
                const size_t cip = IDX(i + 1, j, k), cim = IDX(i - 1, j, k);
                const size_t cjp = IDX(i, j + 1, k), cjm = IDX(i, j - 1, k);
                const size_t ckp = IDX(i, j, ke), ckm = IDX(i, j, kw);
                const double rm = G->rad[i];
                const double exp_rm = 1.0;
                double sinthe = sin(G->the[j]);
                if (sinthe == 0.0) sinthe = 1.0e-5;
                const double costhe = cos(G->the[j]);
                const double cotanthe = costhe / sinthe;
                const double inv_rm = 1.0 / rm;
                const double rmsinthe = rm * sinthe;
                const double inv_2dr = 1.0 / (2.0 * P->dr);
                const double inv_2dthe = 1.0 / (2.0 * P->dthe);
                const double inv_2dphi = 1.0 / (2.0 * P->dphi);
                const double inv_rm2dthe = inv_2dthe / rm;
                const double inv_rmsinthe2dphi = inv_2dphi / rmsinthe;

                const double dudr = (U[cip] - U[cim]) * inv_2dr * exp_rm;
                const double dvdr = (V[cip] - V[cim]) * inv_2dr * exp_rm;
                const double dwdr = (W[cip] - W[cim]) * inv_2dr * exp_rm;
                const double dudthe = (U[cjp] - U[cjm]) * inv_rm2dthe;
                const double dvdthe = (V[cjp] - V[cjm]) * inv_rm2dthe;
                const double dwdthe = (W[cjp] - W[cjm]) * inv_rm2dthe;
                const double dudphi = (U[ckp] - U[ckm]) * inv_rmsinthe2dphi;
                const double dvdphi = (V[ckp] - V[ckm]) * inv_rmsinthe2dphi;
                const double dwdphi = (W[ckp] - W[ckm]) * inv_rmsinthe2dphi;

                const int nb = sol[cim], njm = sol[cjm], njp = sol[cjp], nkm = sol[ckm], nkp = sol[ckp];
                const double tk0 = TK[c], ds0 = DS[c];
                const double tke_im1 = nb ? tk0 : TK[cim], dis_im1 = nb ? ds0 : DS[cim];
                const double tke_jm1 = njm ? tk0 : TK[cjm], tke_jp1 = njp ? tk0 : TK[cjp];
                const double dis_jm1 = njm ? ds0 : DS[cjm], dis_jp1 = njp ? ds0 : DS[cjp];
                const double tke_km1 = nkm ? tk0 : TK[ckm], tke_kp1 = nkp ? tk0 : TK[ckp];
                const double dis_km1 = nkm ? ds0 : DS[ckm], dis_kp1 = nkp ? ds0 : DS[ckp];
                const double dtkedr = (TK[cip] - tke_im1) * inv_2dr * exp_rm;
                const double ddisdr = (DS[cip] - dis_im1) * inv_2dr * exp_rm;
                const double dtkedthe = (tke_jp1 - tke_jm1) * inv_rm2dthe;
                const double ddisdthe = (dis_jp1 - dis_jm1) * inv_rm2dthe;
                const double dtkedphi = (tke_kp1 - tke_km1) * inv_rmsinthe2dphi;
                const double ddisdphi = (dis_kp1 - dis_km1) * inv_rmsinthe2dphi;
                /* passed to the model routines, which form their own theta/phi differences */
                (void)dtkedthe; (void)ddisdthe; (void)dtkedphi; (void)ddisdphi;

                double cnue;
                {
                    const double dis_here = dmax(ds0, dis_min);
                    const double tke_here = dmax(tk0, 0.0);
                    cnue = (model == ATJUP_TURB_K_EPSILON) ? C_nue * tke_here * tke_here / dis_here
                                                           : tke_here / dis_here;
                    cnue = dmin(cnue, nue_max);
                }
                const int curv = PH->turb_curv;
                const double u_r = curv ? U[c] * inv_rm : 0.0;
                const double v_r = curv ? V[c] * inv_rm : 0.0;
                const double w_r = curv ? W[c] * inv_rm : 0.0;
                const double v_cot_r = v_r * cotanthe;
                const double w_cot_r = w_r * cotanthe;
                const double g_rr = dudr, g_rt = dudthe - v_r, g_rp = dudphi - w_r;
                const double g_tr = dvdr, g_tt = dvdthe + u_r, g_tp = dvdphi - w_cot_r;
                const double g_pr = dwdr, g_pt = dwdthe, g_pp = dwdphi + u_r + v_cot_r;
                const double der = 0.66667 * (g_rr + g_tt + g_pp);
                X->prod[c] = dmax(0.0,
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

                if (model == ATJUP_TURB_K_EPSILON) {                      /* 886-927 */
                    const double C_eps_1 = 1.35, C_eps_2 = 1.80;
                    const double y_phys = PH->turb_free ? 1.0e20 : dmax(HM(i) - y_mount, L_m);
                    const double y_star = y_phys / L_m;
                    X->nue_out[c] = C_nue * tk0 * tk0 / dmax(ds0, dis_min);
                    const double d_plus = y_phys * X->vel_star[(size_t)j * km + k] / nue_air;
                    const double f_nue = 1.0 - exp(-0.0115 * d_plus);
                    const double Re_T = tk0 * tk0 * P->u_0 * L_m / dmax(ds0 * nue_air, dis_min * nue_air);
                    const double f_2 = 1.0 - 0.4 / 1.8 * exp(-Re_T * Re_T / 36.0);
                    X->nue_out[c] *= f_nue;
                    const double y_star2 = y_star * y_star;
                    const double L_k = -2.0 * tk0 / y_star2;
                    const double L_w = -2.0 * ds0 / y_star2 * exp(-d_plus / 2.0);
                    const double P_k = X->prod[c];
                    const double Y_k = ds0;
                    const double tke_safe = dmax(tk0, dis_min);
                    const double P_w = C_eps_1 * ds0 / tke_safe * P_k;
                    const double Y_w = C_eps_2 * f_2 * ds0 * ds0 / tke_safe;
                    X->tke_source[c] = P_k - Y_k + L_k / PH->re_turb;
                    X->dis_source[c] = P_w - Y_w + L_w / PH->re_turb;
                } else if (model == ATJUP_TURB_K_OMEGA) {                 /* 930-1017 */
                    const double bet_star = 0.09, gam = 0.52, C_lim = 0.875, bet_0 = 0.0708;
                    const double exp_rm_k = 1.0 / (rm + 1.0);
                    const double dtkedr_neu = nb ? (TK[cip] - tk0) * (1.0 / (2.0 * P->dr)) * exp_rm_k : dtkedr;
                    const double ddisdr_neu = nb ? (DS[cip] - ds0) * (1.0 / (2.0 * P->dr)) * exp_rm_k : ddisdr;
                    const double dtkedthe_neu = (tke_jp1 - tke_jm1) / (rm * 2.0 * P->dthe);
                    const double ddisdthe_neu = (dis_jp1 - dis_jm1) / (rm * 2.0 * P->dthe);
                    const double dtkedphi_neu = (tke_kp1 - tke_km1) / (rmsinthe * 2.0 * P->dphi);
                    const double ddisdphi_neu = (dis_kp1 - dis_km1) / (rmsinthe * 2.0 * P->dphi);
                    const double dudr_k = (U[cip] - U[cim]) / (2.0 * P->dr) / (rm + 1.0);
                    const double dvdthe_k = (V[cjp] - V[cjm]) / (rm * 2.0 * P->dthe);
                    const double dwdphi_k = (W[ckp] - W[ckm]) / (rmsinthe * 2.0 * P->dphi);
                    const double dudthe_u = (U[cjp] - U[cjm]) / (rm * 2.0 * P->dthe);
                    const double dudphi_u = (U[ckp] - U[ckm]) / (rmsinthe * 2.0 * P->dphi);
                    const double dvdr_u = (V[cip] - V[cim]) / (2.0 * P->dr) / (rm + 1.0);
                    const double dwdr_u = (W[cip] - W[cim]) / (2.0 * P->dr) / (rm + 1.0);
                    const double dvdphi_u = (V[ckp] - V[ckm]) / (rmsinthe * 2.0 * P->dphi);
                    const double dwdthe_u = (W[cjp] - W[cjm]) / (rm * 2.0 * P->dthe);
                    const double S11 = dudr_k, S22 = dvdthe_k, S33 = dwdphi_k;
                    const double S12 = 0.5 * (dudthe_u + dvdr_u);
                    const double S13 = 0.5 * (dudphi_u + dwdr_u);
                    const double S23 = 0.5 * (dvdphi_u + dwdthe_u);
                    const double S_mag = sqrt(2.0 * (S11 * S11 + S22 * S22 + S33 * S33
                                                     + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23)));
                    const double w_hat = dmax(ds0, C_lim * S_mag / sqrt(bet_star));
                    double sig_d = dtkedr_neu * ddisdr_neu + dtkedthe_neu * ddisdthe_neu + dtkedphi_neu * ddisdphi_neu;
                    sig_d = (sig_d <= 0.0) ? 0.0 : 0.125;
                    const double chi_w = fabs(Omega * Omega * S_mag / pow(bet_star * dmax(ds0, 1.0e-20), 3));
                    const double f_bet = (1.0 + 85.0 * chi_w) / (1.0 + 100.0 * chi_w);
                    const double bet_wc = bet_0 * f_bet;
                    X->nue_out[c] = tk0 / dmax(w_hat, 1.0e-20);
                    const double P_k = dmin(X->prod[c], 20.0 * bet_star * tk0 * ds0);
                    const double Y_k = bet_star * tk0 * ds0;
                    const double P_w = gam * ds0 / dmax(tk0, 1.0e-20) * P_k;
                    const double Y_w = bet_wc * ds0 * ds0;
                    const double D_w = sig_d / dmax(ds0, 1.0e-20)
                        * (dtkedr_neu * ddisdr_neu + dtkedthe_neu * ddisdthe_neu + dtkedphi_neu * ddisdphi_neu);
                    X->tke_source[c] = P_k - Y_k;
                    X->dis_source[c] = P_w - Y_w + D_w;
                } else {                                                  /* 1021-1106 */
                    const double a1 = 0.31, bet_star = 0.09, bet1 = 0.0333, bet2 = 0.0368;
                    const double gam1 = 0.413, gam2 = 0.2, sig_w2 = 1.168;
                    const double nue_air_nd = nue_air / (P->u_0 * L_m);
                    const double dz_layer = dmax(1.0, layer_dz_m(X, im, i - 1 > 0 ? i - 1 : 0));
                    const double y_phys = PH->turb_free ? 1.0e20 : dmax(HM(i) - y_mount, dz_layer);
                    const double y_star = y_phys / L_m;
                    const double exp_rm_k = 1.0 / (rm + 1.0);
                    const double dtkedr_neu = nb ? (TK[cip] - tk0) * (1.0 / (2.0 * P->dr)) * exp_rm_k : dtkedr;
                    const double ddisdr_neu = nb ? (DS[cip] - ds0) * (1.0 / (2.0 * P->dr)) * exp_rm_k : ddisdr;
                    const double dtkedthe_neu = (tke_jp1 - tke_jm1) / (rm * 2.0 * P->dthe);
                    const double ddisdthe_neu = (dis_jp1 - dis_jm1) / (rm * 2.0 * P->dthe);
                    const double dtkedphi_neu = (tke_kp1 - tke_km1) / (rmsinthe * 2.0 * P->dphi);
                    const double ddisdphi_neu = (dis_kp1 - dis_km1) / (rmsinthe * 2.0 * P->dphi);
                    const double grad_dot = dtkedr_neu * ddisdr_neu + dtkedthe_neu * ddisdthe_neu
                                          + dtkedphi_neu * ddisdphi_neu;
                    const double CD_kw = dmax(2.0 * sig_w2 / dmax(ds0, 1.0e-20) * grad_dot, 1.0e-20);
                    const double dis_safe = dmax(ds0, 1.0e-20);
                    const double arg1 = dmin(
                        dmax(sqrt(tk0) / (bet_star * dis_safe * y_star),
                             500.0 * nue_air_nd / (y_star * y_star * dis_safe)),
                        4.0 * sig_w2 * tk0 / (CD_kw * y_star * y_star));
                    const double arg2 = dmax(
                        2.0 * sqrt(tk0) / (bet_star * dis_safe * y_star),
                        500.0 * nue_air_nd / (y_star * y_star * dis_safe));
                    const double F1 = tanh(pow(arg1, 4));
                    const double F2 = tanh(pow(arg2, 2));
                    X->nue_out[c] = a1 * tk0 / dmax(a1 * dis_safe, Omega * F2);
                    const double tke_safe = dmax(tk0, 1.0e-20);
                    const double P_k = dmin(X->prod[c], 20.0 * bet_star * tke_safe * dis_safe);
                    const double Y_k = bet_star * tke_safe * dis_safe;
                    const double P_w = (F1 * gam1 + (1.0 - F1) * gam2) * P_k * dis_safe / tke_safe;
                    const double Y_w = (F1 * bet1 + (1.0 - F1) * bet2) * dis_safe * dis_safe;
                    const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_safe * grad_dot;
                    X->tke_source[c] = P_k - Y_k;
                    X->dis_source[c] = P_w - Y_w + D_w;
                }
                if (PH->turb_buoy != 0) {                                 /* 843-867, buoy 1 or 2 */
                    const double Pr_t = 0.9;
                    const double T = S->t[c] * P->t_ref;
                    const double dz = HM(i + 1) - HM(i - 1);
                    const double dTdz = (S->t[cip] - S->t[cim]) * P->t_ref / dz;
                    const double Gam = P->g / P->cp_mix, fac = 1.0;
                    const double N2 = (T > 0.0 && dz > 0.0) ? P->g / T * (dTdz + Gam) * fac : 0.0;
                    if (isfinite(N2) && (N2 > 0.0 || PH->turb_buoy == 2)) {
                        const double tL = L_m / P->u_0;
                        X->tke_source[c] -= dmax(0.0, X->nue_out[c]) * N2 * tL * tL / Pr_t;
                    }
                }
            }
        }
    /* clamp-out pass */
    for (int j = 1; j < jm - 1; j++)
        for (int k = 0; k < km - 1; k++) {
            const double vs = X->vel_star[(size_t)j * km + k];
            const double k_bg_nd = PH->turb_free ? PH->turb_k_bg / (P->u_0 * P->u_0)
                                 : 0.01 * vs * vs / (sqrt(C_nue) * P->u_0 * P->u_0);
            for (int i = 1; i < im - 1; i++) {
                const size_t c = IDX(i, j, k);
                if (sol[c]) continue;
                TK[c] = dmax(k_bg_nd, TK[c]);
                DS[c] = dmax(dis_min, DS[c]);
                X->nue_out[c] = clamp3(X->nue_out[c], 0.0, nue_max);
                const double dis_src_max = 20.0 * DS[c] * DS[c];
                X->dis_source[c] = clamp3(X->dis_source[c], -dis_src_max, dis_src_max);
                const double tke_src_max = 20.0 * TK[c] * DS[c];
                X->tke_source[c] = clamp3(X->tke_source[c], -tke_src_max, tke_src_max);
            }
        }
    ora_turb_wall_bc(P, PH, G, X);
    /* zero_land_cells */
    for (size_t c = 0; c < N; c++)
        if (sol[c]) {
            TK[c] = 0.0; X->tken[c] = 0.0; DS[c] = 0.0; X->disn[c] = 0.0;
            X->nue_out[c] = 0.0; X->prod[c] = 0.0; X->tke_source[c] = 0.0; X->dis_source[c] = 0.0;
        }
    /* clamp_nue */
    {
        int i_abl = 0;
        while (i_abl < im - 1 && HM(i_abl) <= PH->abl_height) i_abl++;
        const double taper_dz = dmax(1.0, HM(i_abl < im - 1 ? i_abl : im - 1) - HM(i_abl - 1 > 0 ? i_abl - 1 : 0));
        for (int i = 0; i < im; i++)
            for (int j = 0; j < jm; j++)
                for (int k = 0; k < km; k++) {
                    double f = 1.0;
                    if (PH->abl_taper) {
                        const double z_agl = HM(i) - HM(G->topo[(size_t)j * km + k]);
                        f = clamp3((PH->abl_height + taper_dz - z_agl) / taper_dz, 0.0, 1.0);
                    }
                    const size_t c = IDX(i, j, k);
                    X->nue_out[c] = clamp3(X->nue_out[c], 0.0, nue_max) * f;
                }
    }
    /* seam_copy */
    double* eight[8] = {TK, DS, X->tken, X->disn, X->nue_out, X->prod, X->tke_source, X->dis_source};
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            for (int q = 0; q < 8; q++) eight[q][IDX(i, j, km - 1)] = eight[q][IDX(i, j, 0)];
    /* fill_lid_corners (TURB_FREE, bc_turb_active() false on ATJUP) */
    if (PH->turb_free) {
        const int il = im - 1;
        for (int j = 1; j < jm - 1; j++)
            for (int k = 0; k < km; k++)
                for (int q = 0; q < 8; q++) eight[q][IDX(il, j, k)] = eight[q][IDX(il - 1, j, k)];
        for (int i = 0; i < im; i++)
            for (int k = 0; k < km; k++)
                for (int q = 0; q < 8; q++) {
                    eight[q][IDX(i, 0, k)] = eight[q][IDX(i, 1, k)];
                    eight[q][IDX(i, jm - 1, k)] = eight[q][IDX(i, jm - 2, k)];
                }
    }
    ora_turb_wall_omega(P, PH, G, X);
#undef HM
}

/* ---------------------------------------------------------------------------------------------
 * The loop's microphysics: radiation, precipitation, the NH4SH equilibrium, the chemistry fluxes
 * and the species clamp. Operand order as in the reference throughout.
 * ------------------------------------------------------------------------------------------- */

/* Radiation.h:251-456: per (j, k) column from the first fluid level to the top, layer optical
 * depths of collision-induced H2 absorption, CH4/NH3 bands and clouds, the grey downward and
 * upward thermal fluxes, the shortwave attenuated by pressure, and the heating of each layer. */
void ora_radiation(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G, ora_state* S,
                   ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    const double t_ref = P->t_ref, g = P->g;
    const double sigma = 5.670374419e-8, P0_phys = 1.0e5, he_ratio = 0.6, C_cia = 3.5e-6;
    const double kappa_ch4 = 0.003, kappa_nh3 = 1.5, kappa_cloud = 25.0, kappa_ice = 12.0;
    const double tau_cloud_cap = 0.4, opac_cal = 0.025;
    const double pi_ = 3.14159265358979323846;
    const double comp = MC->x_H2 * MC->x_H2 + he_ratio * MC->x_H2 * MC->x_He;
    const double cia_coeff = C_cia * MC->cia_strength * comp / g;
    const double opac_mult = MC->opacity_strength;
    double B[128], eps[128], Fd[130], Fu[130], Fsw[130];
    if (im > 127) return;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            int i_base = G->topo[(size_t)j * km + k];
            if (i_base < 0) i_base = 0;
            const int i_top = im - 1;
            if (i_base >= i_top) continue;
            for (int i = i_base; i <= i_top; i++) {
                const size_t c = IDX(i, j, k);
                const double T = S->t[c] * t_ref;
                B[i] = sigma * T * T * T * T;
                const double P_lo = S->p_stat[c] * P0_phys;
                const double P_hi = (i < i_top) ? S->p_stat[IDX(i + 1, j, k)] * P0_phys : 0.0;
                double dP = P_lo - P_hi;
                if (dP < 0.0) dP = 0.0;
                const double P_mean = 0.5 * (P_lo + P_hi);
                const double dm = dP / g;
                const double tau_cia = (T > 0.0) ? cia_coeff * (P_mean / T) * dP : 0.0;
                const double rho_c = S->rho_mix[c];
                const double inv_rho = (rho_c > 0.0 && isfinite(rho_c)) ? 1.0 / rho_c : 0.0;
                const double q_ch4 = dmax(0.0, X->q[ATJUP_S_CH4][c]) * inv_rho;
                const double q_nh3 = dmax(0.0, X->q[ATJUP_S_NH3][c]) * inv_rho;
                const double tau_gas = opac_mult * opac_cal * (kappa_ch4 * q_ch4 + kappa_nh3 * q_nh3) * dm;
                const double q_liq = (dmax(0.0, X->q[ATJUP_S_H2O_CLOUD][c])
                                    + dmax(0.0, X->q[ATJUP_S_NH3_CLOUD][c])
                                    + dmax(0.0, X->q[ATJUP_S_CH4_CLOUD][c])) * inv_rho;
                const double q_ice = (dmax(0.0, X->q[ATJUP_S_H2O_ICE][c])
                                    + dmax(0.0, X->q[ATJUP_S_NH3_ICE][c])
                                    + dmax(0.0, X->q[ATJUP_S_CH4_ICE][c])) * inv_rho;
                double tau_cloud = opac_mult * opac_cal * (kappa_cloud * q_liq + kappa_ice * q_ice) * dm;
                if (tau_cloud > tau_cloud_cap) tau_cloud = tau_cloud_cap;
                const double tau_l = tau_cia + tau_gas + tau_cloud;
                eps[i] = 1.0 - exp(-tau_l);
            }
            for (int i = 0; i <= im + 1; i++) Fsw[i] = 0.0;
            if (MC->solar_on != 0) {
                const double colat = pi_ * (double)j / (double)(jm - 1);
                const double cos_lat = dmax(0.0, sin(colat));
                const double F_sun_toa = MC->solar_strength * MC->S_solar * (1.0 - MC->albedo_bond) * cos_lat / pi_;
                for (int i = i_base; i <= i_top + 1; i++) {
                    const double p_bar = (i <= i_top) ? S->p_stat[IDX(i, j, k)] : 0.0;
                    Fsw[i] = F_sun_toa * exp(-MC->sw_tau_per_bar * dmax(0.0, p_bar));
                }
            }
            Fd[i_top + 1] = 0.0;
            for (int i = i_top; i >= i_base; i--) Fd[i] = Fd[i + 1] * (1.0 - eps[i]) + eps[i] * B[i];
            if (MC->rad_bottom == 1) Fu[i_base] = dmax(0.0, 2.0 * B[i_base] - Fd[i_base + 1]);
            else Fu[i_base] = Fd[i_base] + MC->F_int + Fsw[i_base];
            for (int i = i_base; i <= i_top; i++) Fu[i + 1] = Fu[i] * (1.0 - eps[i]) + eps[i] * B[i];
            for (int i = i_base; i <= i_top; i++) {
                const double net_bot = Fu[i] - Fd[i];
                const double net_top = Fu[i + 1] - Fd[i + 1];
                double dz = (i < i_top) ? layer_dz_m(X, im, i) : layer_dz_m(X, im, i - 1);
                if (dz <= 0.0) dz = 1.0;
                const double sw_absorbed = Fsw[i + 1] - Fsw[i];
                const double Q_sw = sw_absorbed / dz;
                S->Q_rad[IDX(i, j, k)] = (net_bot - net_top) / dz + Q_sw;
            }
            for (int i = 0; i < i_base; i++) S->Q_rad[IDX(i, j, k)] = 0.0;
        }
}

/* Precipitation.h:273-445 for one species (gas q: 0 H2O, 1 NH3, 2 CH4). */
static void precip_column(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G,
                          ora_state* S, ora_phys* X, int q) {
    const int im = P->im, jm = P->jm, km = P->km;
    const AtjupGasParams* gs = &MC->gas[q];
    const int sv = q == 0 ? ATJUP_S_H2O : (q == 1 ? ATJUP_S_NH3 : ATJUP_S_CH4);
    double *vap = X->q[sv], *cld = X->q[sv + 1], *ice = X->q[sv + 2];
    double *Sv = (double*)X->s_precip[3 * q], *Sc = (double*)X->s_precip[3 * q + 1];
    double *Si = (double*)X->s_precip[3 * q + 2];
    const double t_ref = P->t_ref;
    const double Lf = gs->ls - gs->lv;
    const double P_max_flux = 1.0e-4, dep_frac = 1.0, ratio_cap = 5.0, rs = MC->precip_rate_scale;
    const double c_c_au = 2.0e-8, c_i_au = 5.0e-8, q_c_crit = 5.0e-4, c_ac = 1.0e-7;
    const double c_rim = 1.0e-8, z_csg = 2.5e-8, a_ev = 2.76e-3, c_melt_K = 0.2, c_frz_K = 0.2;
    const double P_ref = 1.0e-4, v_fall = 2.0;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            int i_base = G->topo[(size_t)j * km + k];
            if (i_base < 0) i_base = 0;
            const int i_top = im - 1;
            if (i_base >= i_top) continue;
            double Pr = 0.0, Ps = 0.0, Pg = 0.0;   /* the fluxes leaving the layer above */
            for (int i = i_top - 1; i >= i_base; i--) {
                const size_t c = IDX(i, j, k);
                const double T = S->t[c] * t_ref;
                const double p_u = S->p_stat[c];
                const double q_v = dmax(0.0, vap[c]), q_c = dmax(0.0, cld[c]), q_i = dmax(0.0, ice[c]);
                const double E_r = ora_svp(T, gs->C, gs->L0, gs->R, gs->del_alf, gs->del_bet);
                double rho = P->r_mix;
                if (P->local_rho && S->rho_mix[c] > 0.0 && isfinite(S->rho_mix[c])) rho = S->rho_mix[c];
                const double q_sat = (p_u > E_r) ? rho * gs->ep * E_r / p_u : q_v;
                const double dz = dmax(0.0, layer_dz_m(X, im, i));
                if (dz <= 0.0) continue;   /* the fluxes pass through unchanged */
                const double F_r_in = Pr, F_s_in = Ps, F_g_in = Pg;
                const double Rain = dmin(ratio_cap, F_r_in / P_ref);
                const double Snow = dmin(ratio_cap, F_s_in / P_ref);
                const double Graupel = dmin(ratio_cap, F_g_in / P_ref);
                const double Rain_79 = (Rain > 0.0) ? pow(Rain, 7.0 / 9.0) : 0.0;
                const double Rain_49 = (Rain > 0.0) ? pow(Rain, 4.0 / 9.0) : 0.0;
                const int warm = (T >= gs->t_0);
                const double S_c_au = (warm && q_c > q_c_crit) ? (rs * c_c_au) * (q_c - q_c_crit) : 0.0;
                const double S_i_au = (!warm && T >= gs->t_00) ? (rs * c_i_au) * q_i : 0.0;
                const double S_ac = warm ? (rs * c_ac) * q_c * Rain_79 : 0.0;
                const double S_s_rim = !warm ? (rs * c_rim) * q_c * Snow : 0.0;
                const double S_g_rim = !warm ? (rs * c_rim) * q_c * Graupel : 0.0;
                const double S_csg = (!warm && q_c > q_c_crit) ? (rs * z_csg) * q_c * Snow : 0.0;
                const double f_melt = warm ? dmin(1.0, c_melt_K * (T - gs->t_0)) : 0.0;
                const double f_frz = warm ? 0.0 : dmin(1.0, c_frz_K * (gs->t_0 - T));
                const double F_s_melt = f_melt * F_s_in, F_g_melt = f_melt * F_g_in;
                const double F_r_frz = f_frz * F_r_in;
                const double F_r_avail = dmax(0.0, F_r_in - F_r_frz + F_s_melt + F_g_melt
                                                   + (S_c_au + S_ac) * dz);
                const double S_ev_raw = (warm && Rain > 0.0 && q_v < q_sat)
                                      ? a_ev * (q_sat - q_v) * Rain_49 : 0.0;
                const double F_ev_sat = dmax(0.0, q_sat - q_v) * v_fall;
                const double F_ev = dmin(dmin(S_ev_raw * dz, F_r_avail), F_ev_sat);
                const double S_ev = F_ev / dz;
                S->Q_precip[c] += Lf * (S_s_rim + S_g_rim + S_csg)
                                + Lf * (F_r_frz - F_s_melt - F_g_melt) / dz
                                - gs->lv * F_ev / dz;
                const double tau = dz / v_fall;
                const double d_c = dmin(dep_frac * q_c, (S_c_au + S_ac + S_s_rim + S_g_rim + S_csg) * tau);
                const double d_i = dmin(dep_frac * q_i, S_i_au * tau);
                if (MC->precip_coupling_on) {
                    const double nd = (P->L_atm * 1.0e3) / P->u_0;
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
        }
}

void ora_precipitation(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G,
                       ora_state* S, ora_phys* X) {
    const size_t N = (size_t)P->im * P->jm * P->km;
    for (size_t c = 0; c < N; c++) {
        S->Q_precip[c] = 0.0;
        for (int q = 0; q < 9; q++) ((double*)X->s_precip[q])[c] = 0.0;
    }
    for (int q = 0; q < 3; q++) precip_column(P, MC, G, S, X, q);
}

/* ChemistryJup.h:291-373 (loop mode): per fluid cell, the extent x of NH3 + H2S -> NH4SH that
 * brings p_NH3 p_H2S to K_p(T) with the latent heat of formation, by bisection. */
void ora_nh4sh_eq(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G, ora_state* S,
                  ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    const double R_univ = 8314.46, atm = 101325.0;
    const double L_f = 4705.0 * log(10.0) * 8314.46 / 51.1114;
    double *nh3 = X->q[ATJUP_S_NH3], *h2s = X->q[ATJUP_S_H2S], *nh4sh = X->q[ATJUP_S_NH4SH];
    /* each cell reads and writes only itself: parallel, bit-identical to one thread */
    #pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++)
            for (int i = 0; i < im; i++) {
                const size_t c = IDX(i, j, k);
                if (G->solid[c]) continue;
                const double T0 = S->t[c] * P->t_ref;
                if (!(T0 > 0.0)) continue;
                double rho = S->rho_mix[c];
                if (!(rho > 0.0) || !isfinite(rho)) rho = P->r_mix;
                const double a = dmax(0.0, nh3[c]) / MC->m_nh3;
                const double b = dmax(0.0, h2s[c]) / MC->m_h2s;
                const double s = dmax(0.0, nh4sh[c]) / MC->m_nh4sh;
                const double heat = L_f * MC->m_nh4sh / (P->cp_mix * rho);
#define KP_(T_) (pow(10.0, 14.82 - 4705.0 / (T_)) * atm * atm)
#define F_(x_) ((a - (x_)) * (b - (x_)) * (R_univ * (T0 + heat * (x_))) * (R_univ * (T0 + heat * (x_))) - KP_(T0 + heat * (x_)))
                const double f0 = F_(0.0);
                double lo, hi;
                if (f0 > 0.0) { lo = 0.0; hi = dmin(a, b); }
                else if (s > 0.0) {
                    if (F_(-s) <= 0.0) { lo = hi = -s; }
                    else { lo = -s; hi = 0.0; }
                } else continue;
                if (hi > lo)
                    for (int it = 0; it < 80; it++) {
                        const double xm = 0.5 * (lo + hi);
                        if (F_(xm) > 0.0) lo = xm; else hi = xm;
                        if (hi - lo <= 1.0e-15 * dmax(a, dmax(b, s))) break;
                    }
#undef F_
#undef KP_
                const double x = (f0 > 0.0) ? lo : hi;
                if (x == 0.0) continue;
                nh3[c] = dmax(0.0, nh3[c] - MC->m_nh3 * x);
                h2s[c] = dmax(0.0, h2s[c] - MC->m_h2s * x);
                nh4sh[c] = dmax(0.0, nh4sh[c] + MC->m_nh4sh * x);
                const double dT = heat * x;
                S->t[c] = (T0 + dT) / P->t_ref;
            }
}

/* ChemistryJup.h:756-780: the spherical Laplacian of the diffusive mass fluxes, with the polar
 * floor on sin(theta) in the metric terms. */
static double chem_laplacian(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G,
                             const double* c, int i, int j, int k) {
    const int jm = P->jm, km = P->km;
    const double rm = G->rad[i];
    const double exp_rm = 1.0, exp_2_rm = exp_rm * exp_rm;
    const double sinthe = sin(G->the[j]);
    const double costhe = cos(G->the[j]);
    const double rmsinthe = rm * dmax(sinthe, MC->polar_divisor_floor);
    const double c0 = c[IDX(i, j, k)];
    const double d2cdr2 = (c[IDX(i + 1, j, k)] - 2.0 * c0 + c[IDX(i - 1, j, k)]) / (P->dr * P->dr) * exp_2_rm;
    const double d2cdthe2 = (c[IDX(i, j + 1, k)] - 2.0 * c0 + c[IDX(i, j - 1, k)]) / (P->dthe * P->dthe);
    const int kw = phi_wrap(1, k - 1, km), ke = phi_wrap(1, k + 1, km);
    const double d2cdphi2 = (c[IDX(i, j, ke)] - 2.0 * c0 + c[IDX(i, j, kw)]) / (P->dphi * P->dphi);
    const double dcdr = (c[IDX(i + 1, j, k)] - c[IDX(i - 1, j, k)]) / (2.0 * P->dr) * exp_rm;
    const double dcdthe = (c[IDX(i, j + 1, k)] - c[IDX(i, j - 1, k)]) / (2.0 * P->dthe);
    return d2cdr2 + 2.0 / rm * dcdr + d2cdthe2 / (rm * rm) + costhe / (rm * rmsinthe) * dcdthe
         + d2cdphi2 / (rmsinthe * rmsinthe);
}

static double superbee_phi(double r) {                /* FluxLimiter.h TVD::superbee_phi */
    return dmax(0.0, dmax(dmin(2.0 * r, 1.0), dmin(r, 2.0)));
}

void ora_chemistry(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G, ora_state* S,
                   ora_phys* X) {
    const int im = P->im, jm = P->jm, km = P->km;
    const uint8_t* sol = G->solid;
    double* spec[3] = {X->q[ATJUP_S_H2S], X->q[ATJUP_S_NH3], X->q[ATJUP_S_NH4SH]};
    const double D[3] = {MC->D_h2s, MC->D_nh3, MC->D_nh4sh};
    double* mf[3] = {(double*)X->massflux_h2s, (double*)X->massflux_nh3, (double*)X->massflux_nh4sh};
    /* DiffMassFluxJup (ChemistryJup.h:375-538): only difflux reaches the dynamics */
    for (int k = 0; k < km - 1; k++)
        for (int j = 1; j < jm - 1; j++)
            for (int i = 1; i < im - 1; i++) {
                const size_t c = IDX(i, j, k);
                if (!(S->t[c] > 0.0) || sol[c]) {
                    for (int q = 0; q < 3; q++) X->difflux[q][c] = 0.0;
                    continue;
                }
                for (int q = 0; q < 3; q++) X->difflux[q][c] = D[q] * chem_laplacian(P, MC, G, spec[q], i, j, k);
            }
    for (int q = 0; q < 3; q++) ora_shapiro(P, G, X->difflux[q], 2, 1.0, 1, 1);
    /* ChemMassRateJup (59-281): massflux = reaction rate + difflux; the rate is 0 with the
     * equilibrium on (ATJUP_NH4SH_EQ=1) and outside the [t_00_nh4sh, t_0_nh4sh] window */
    for (int i = 0; i < im; i++)
        for (int k = 0; k < km; k++) {
            for (int j = 0; j < 3; j++)
                for (int q = 0; q < 3; q++) mf[q][IDX(i, j, k)] = 0.0;
            for (int j = jm - 3; j < jm; j++)
                for (int q = 0; q < 3; q++) mf[q][IDX(i, j, k)] = 0.0;
        }
    for (int k = 0; k < km - 1; k++)
        for (int j = 3; j < jm - 3; j++)
            for (int i = 1; i < im - 1; i++) {
                const size_t c = IDX(i, j, k);
                if (sol[c] && sol[IDX(i - 1, j, k)] && sol[IDX(i + 1, j, k)] && sol[IDX(i, j - 1, k)]
                    && sol[IDX(i, j + 1, k)] && sol[IDX(i, j, phi_wrap(1, k - 1, km))]
                    && sol[IDX(i, j, phi_wrap(1, k + 1, km))]) {
                    for (int q = 0; q < 3; q++) mf[q][c] = 0.0;
                    continue;
                }
                double w[3] = {0.0, 0.0, 0.0};    /* H2S, NH3, NH4SH */
                const double t_u = S->t[c] * P->t_ref;
                if (!MC->nh4sh_eq && t_u <= MC->t_0_nh4sh && t_u >= MC->t_00_nh4sh) {
                    /* kf = A T^B exp(-T_d / T), A 15000, B -0.5, T_d 3020 (react_rate_const);
                     * kb = kf / keq, keq = m_nh4sh / (m_nh3 m_h2s) */
                    const double keq = MC->m_nh4sh / (MC->m_nh3 * MC->m_h2s);
                    const double kf = 15000.0 * pow(t_u, -0.5) * exp(-3020.0 / t_u);
                    const double kb = kf / keq;
                    const double nh3 = spec[1][c], h2s = spec[0][c], nh4sh = spec[2][c];
                    /* concentrations scaled so that they sum to r_mix (the default normalisation) */
                    const double sum_c = nh3 / MC->m_nh3 + h2s / MC->m_h2s + nh4sh / MC->m_nh4sh;
                    const double denom = (sum_c == 0.0) ? 0.0 : P->r_mix / sum_c;
                    const double c_nh3 = nh3 / MC->m_nh3 * denom;
                    const double c_h2s = h2s / MC->m_h2s * denom;
                    const double c_nh4sh = nh4sh / MC->m_nh4sh * denom;
                    const double R_diff = kf * c_nh3 * c_h2s - kb * c_nh4sh;
                    w[0] = -MC->m_h2s * R_diff;
                    w[1] = -MC->m_nh3 * R_diff;
                    w[2] = MC->m_nh4sh * R_diff;
                }
                for (int q = 0; q < 3; q++) mf[q][c] = w[q] + X->difflux[q][c];
            }
    /* FluxLimiter<cJupiterModel>::nh4sh (FluxLimiter.h): superbee anti-diffusion of NH4SH */
    const double* Q = X->q[ATJUP_S_NH4SH];
    double* fl = (double*)X->fluxlim_nh4sh;
    const double eps = 1.0e-12;
    for (int k = 0; k < km - 1; k++)
        for (int j = 1; j < jm - 1; j++)
            for (int i = 1; i < im - 1; i++) {
                const size_t c = IDX(i, j, k);
                const double q = Q[c];
                const double q_rp = Q[IDX(i + 1, j, k)], q_rm = Q[IDX(i - 1, j, k)];
                const double q_tp = Q[IDX(i, j + 1, k)], q_tm = Q[IDX(i, j - 1, k)];
                const double q_pp = Q[IDX(i, j, phi_wrap(1, k + 1, km))];
                const double q_pm = Q[IDX(i, j, phi_wrap(1, k - 1, km))];
                const double u = S->u[c], v = S->v[c], w = S->w[c];
                const double rm = G->rad[i];
                const double sinthe = dmax(MC->polar_divisor_floor, fabs(sin(G->the[j])));
                const double inv_rm = 1.0 / rm;
                const double inv_rmsinthe = 1.0 / (rm * sinthe);
                double corr = 0.0;
                {
                    const double df = q_rp - q, db = q - q_rm;
                    const double denom = df + (df >= 0.0 ? eps : -eps);
                    const double r = (u >= 0.0) ? db / denom
                                   : ((i + 2 < im ? Q[IDX(i + 2, j, k)] : q_rp) - q_rp) / denom;
                    corr += (1.0 - superbee_phi(r)) * fabs(u) * (df - db) / (2.0 * P->dr);
                }
                {
                    const double df = q_tp - q, db = q - q_tm;
                    const double denom = df + (df >= 0.0 ? eps : -eps);
                    const double q_far = (j + 2 < jm) ? Q[IDX(i, j + 2, k)] : (C43 * q_tp - C13 * q);
                    const double r = (v >= 0.0) ? db / denom : (q_far - q_tp) / denom;
                    corr += (1.0 - superbee_phi(r)) * fabs(v) * inv_rm * (df - db) / (2.0 * P->dthe);
                }
                {
                    const double df = q_pp - q, db = q - q_pm;
                    const double denom = df + (df >= 0.0 ? eps : -eps);
                    const double r = (w >= 0.0) ? db / denom
                                   : (Q[IDX(i, j, phi_wrap(1, k + 2, km))] - q_pp) / denom;
                    corr += (1.0 - superbee_phi(r)) * fabs(w) * inv_rmsinthe * (df - db) / (2.0 * P->dphi);
                }
                fl[c] = corr;
            }
    for (int q = 0; q < 3; q++) ora_shapiro(P, G, mf[q], 2, 1.0, 1, 1);
    ora_shapiro(P, G, fl, 2, 1.0, 1, 1);
}

void ora_clamp_species(const AtjupParams* P, ora_phys* X) {
    const size_t N = (size_t)P->im * P->jm * P->km;
    for (int s = 0; s < ATJUP_S_COUNT; s++)
        for (size_t c = 0; c < N; c++)
            if (!(X->q[s][c] >= 0.0)) X->q[s][c] = 0.0;
}

/* One iteration of the loop with the physics on (cJupiterModel.cpp:1032-1381 with the schedule of
 * the harness: even iterations and the first run the pressure solve, mixture density, radiation,
 * the three saturation adjustments, the NH4SH equilibrium, precipitation, the scalar sync of
 * ATJUP_RK_SCALAR_SYNC = 2, the closure update and the chemistry block; every iteration runs RK4,
 * the boundary passes, the closure's wall law again, the in-loop Shapiro filter, the column
 * balance of v, the species clamp and restoreVar). S->nue must be X->nue_out. */
/* -------------------------------------------------------------------------------------------
 * Moist convective adjustment with the Ledoux criterion (ConvectiveAdjustment.h:403-849, the
 * driver's call at cJupiterModel.cpp:1300-1320) with Jupiter's defaults: no latitude smoothing,
 * the t_0 phase rule, constant cp. Gases H2O and NH3 (MC->gas[0], gas[1]); tracers H2S (a gas in
 * the virtual temperature) and NH4SH (a condensate carrying its heat of formation). The report
 * counters go to stats[8] = {columns, layers, moist triggers, dry triggers, pairs unstable in T,
 * of those held, skipped, most sweeps}; the conservation drift is print-only in the reference.
 * ------------------------------------------------------------------------------------------- */
enum { MCA_NG = 2, MCA_NT = 2, MCA_MAXI = 128, MCA_NITER = 60 };
static const double MCA_TOL_K = 1.0e-7, MCA_TOL_T = 1.0e-10;

typedef struct {
    const AtjupGasParams* g[MCA_NG];
    double tr_ep[MCA_NT], tr_L[MCA_NT];
    int tr_cond[MCA_NT];
    double cp, grav;
    int ledoux, loading;
} mca_ctx;

/* mass fraction at saturation over the phase T selects (ConvectiveAdjustment.h:440-453) */
static double mca_qsat(const mca_ctx* M, int g, double T, double p) {
    const AtjupGasParams* s = M->g[g];
    const double E = (T >= s->t_0) ? ora_svp(T, s->C, s->L0, s->R, s->del_alf, s->del_bet)
                                   : ora_svp(T, s->C_i, s->L0_i, s->R, s->del_alf_i, s->del_bet_i);
    const double q = s->ep * E / p;
    return isfinite(q) ? q : 0.0;
}
static double mca_lat(const mca_ctx* M, int g, double T) {
    return T >= M->g[g]->t_0 ? M->g[g]->lv : M->g[g]->ls;
}
static double mca_fof(const mca_ctx* M, double TT, double hL, const double* qt, double p, double z) {
    double f = M->cp * TT + M->grav * z - hL;
    for (int g = 0; g < MCA_NG; g++) f -= mca_lat(M, g, TT) * dmax(0.0, qt[g] - mca_qsat(M, g, TT, p));
    return f;
}
/* equilibrium temperature of (h_L, q_t) at (p, z) by Illinois regula falsi in the bracket
 * [all vapour, all condensed] (ConvectiveAdjustment.h:459-486) */
static int mca_equil(const mca_ctx* M, double hL, const double* qt, double p, double z, double* T,
                     double* cond) {
    const double T_lo = (hL - M->grav * z) / M->cp;
    if (!(T_lo > 0.0) || !(p > 0.0)) return 0;
    int any = 0;
    for (int g = 0; g < MCA_NG; g++) if (qt[g] > mca_qsat(M, g, T_lo, p)) { any = 1; break; }
    if (!any) {
        *T = T_lo;
        for (int g = 0; g < MCA_NG; g++) cond[g] = 0.0;
        return 1;
    }
    double span = 0.0;
    for (int g = 0; g < MCA_NG; g++) span += dmax(M->g[g]->lv, M->g[g]->ls) * dmax(0.0, qt[g]);
    double a = T_lo, b = T_lo + span / M->cp + 1.0e-9;
    double fa = mca_fof(M, a, hL, qt, p, z), fb = mca_fof(M, b, hL, qt, p, z);
    int side = 0;
    for (int it = 0; it < MCA_NITER && b - a > MCA_TOL_T; it++) {
        double c = (fb - fa != 0.0) ? b - fb * (b - a) / (fb - fa) : 0.5 * (a + b);
        if (!(c > a && c < b)) c = 0.5 * (a + b);
        const double fc = mca_fof(M, c, hL, qt, p, z);
        if (fc < 0.0) { a = c; fa = fc; if (side == -1) fb *= 0.5; side = -1; }
        else          { b = c; fb = fc; if (side == +1) fa *= 0.5; side = +1; }
        if (fabs(fc) <= M->cp * MCA_TOL_T) { a = b = c; break; }
    }
    *T = b;
    for (int g = 0; g < MCA_NG; g++) cond[g] = dmax(0.0, qt[g] - mca_qsat(M, g, *T, p));
    return 1;
}

/* one column's state and the parcel test (ConvectiveAdjustment.h:524-675) */
typedef struct {
    double T[MCA_MAXI], p[MCA_MAXI], z[MCA_MAXI], rho[MCA_MAXI], w[MCA_MAXI], hL[MCA_MAXI];
    double T0[MCA_MAXI], Teq[MCA_MAXI], hL0[MCA_MAXI];
    double qt[MCA_MAXI * MCA_NG], qv[MCA_MAXI * MCA_NG], qc[MCA_MAXI * MCA_NG];
    double qi[MCA_MAXI * MCA_NG], ceq[MCA_MAXI * MCA_NG], qt0[MCA_MAXI * MCA_NG];
    double qr[MCA_MAXI * MCA_NT], qr0[MCA_MAXI * MCA_NT];
    char eq_ok[MCA_MAXI], touched[MCA_MAXI], cen_u[MCA_MAXI], cen_m[MCA_MAXI];
} mca_col;

static double mca_trE(const mca_ctx* M, const mca_col* C, int i) {
    double e = 0.0;
    for (int r = 0; r < MCA_NT; r++) e += M->tr_L[r] * C->qr[i * MCA_NT + r];
    return e;
}
static double mca_tv(const mca_ctx* M, const mca_col* C, double TT, const double* v,
                     const double* cnd, int i) {
    if (!M->ledoux) return TT;
    double f = 1.0;
    for (int g = 0; g < MCA_NG; g++) {
        f += v[g] * (1.0 / M->g[g]->ep - 1.0);
        if (M->loading) f -= cnd[g];
    }
    for (int r = 0; r < MCA_NT; r++) {
        const double q = C->qr[i * MCA_NT + r];
        if (M->tr_ep[r] > 0.0) f += q * (1.0 / M->tr_ep[r] - 1.0);
        else if (M->tr_cond[r] && M->loading) f -= q;
    }
    return TT * f;
}
/* parcel from a lifted to b: unstable when lighter than the air at b in its own equilibrium */
static int mca_unstable(const mca_ctx* M, mca_col* C, int a, int b, int* held, int* moist) {
    double Tp, pc[MCA_NG], pv[MCA_NG], ec[MCA_NG], ev[MCA_NG];
    if (!mca_equil(M, C->hL[a] + mca_trE(M, C, a), &C->qt[a * MCA_NG], C->p[b], C->z[b], &Tp, pc))
        return 0;
    if (!C->eq_ok[b]) {
        if (!mca_equil(M, C->hL[b] + mca_trE(M, C, b), &C->qt[b * MCA_NG], C->p[b], C->z[b],
                       &C->Teq[b], &C->ceq[b * MCA_NG]))
            return 0;
        C->eq_ok[b] = 1;
    }
    const double Tb = C->Teq[b];
    int wet = 0;
    for (int g = 0; g < MCA_NG; g++) {
        ec[g] = C->ceq[b * MCA_NG + g];
        pv[g] = C->qt[a * MCA_NG + g] - pc[g];
        if (pc[g] > 0.0) wet = 1;
        ev[g] = C->qt[b * MCA_NG + g] - ec[g];
    }
    const double dTv = mca_tv(M, C, Tp, pv, pc, a) - mca_tv(M, C, Tb, ev, ec, b);
    if (held) *held = (Tp - Tb > MCA_TOL_K) && !(dTv > MCA_TOL_K);
    if (moist) *moist = wet;
    return dTv > MCA_TOL_K;
}
/* cell q to equilibrium from its h_L and q_t */
static int mca_settle(const mca_ctx* M, mca_col* C, int q) {
    double TT, pc[MCA_NG];
    if (!mca_equil(M, C->hL[q] + mca_trE(M, C, q), &C->qt[q * MCA_NG], C->p[q], C->z[q], &TT, pc))
        return 0;
    C->T[q] = TT;
    C->Teq[q] = TT;
    C->eq_ok[q] = 1;
    for (int g = 0; g < MCA_NG; g++) {
        const int x = q * MCA_NG + g;
        C->ceq[x] = pc[g];
        C->qv[x] = C->qt[x] - pc[g];
        if (TT >= M->g[g]->t_0) { C->qc[x] = pc[g]; C->qi[x] = 0.0; }
        else { C->qi[x] = pc[g]; C->qc[x] = 0.0; }
    }
    C->touched[q] = 1;
    return 1;
}
/* mix h_L, q_t and the tracers over [a, b], mass-weighted, and settle every cell */
static int mca_mix(const mca_ctx* M, mca_col* C, int a, int b) {
    double sw = 0.0, sh = 0.0, sq[MCA_NG] = {0.0}, sr[MCA_NT] = {0.0};
    for (int q = a; q <= b; q++) {
        sw += C->w[q];
        sh += C->w[q] * C->hL[q];
        for (int g = 0; g < MCA_NG; g++) sq[g] += C->w[q] * C->qt[q * MCA_NG + g];
        for (int r = 0; r < MCA_NT; r++) sr[r] += C->w[q] * C->qr[q * MCA_NT + r];
    }
    for (int q = a; q <= b; q++) {
        C->hL[q] = sh / sw;
        for (int g = 0; g < MCA_NG; g++) C->qt[q * MCA_NG + g] = sq[g] / sw;
        for (int r = 0; r < MCA_NT; r++) C->qr[q * MCA_NT + r] = sr[r] / sw;
        if (!mca_settle(M, C, q)) return 0;
    }
    return 1;
}

void ora_mca(const AtjupParams* P, const AtjupMicro* MC, const AtjupMca* A, const ora_grid* G,
             ora_state* S, ora_phys* X, int64_t* stats) {
    const int im = P->im, jm = P->jm, km = P->km;
    mca_ctx M;
    M.g[0] = &MC->gas[0];
    M.g[1] = &MC->gas[1];
    M.tr_ep[0] = A->ep_h2s; M.tr_cond[0] = 0; M.tr_L[0] = 0.0;     /* H2S   */
    M.tr_ep[1] = 0.0;       M.tr_cond[1] = 1; M.tr_L[1] = A->L_nh4sh;   /* NH4SH */
    M.cp = P->cp_mix;
    M.grav = P->g;
    M.ledoux = A->ledoux;
    M.loading = A->loading;
    const double relax = dmin(1.0, dmax(0.0, A->relax));
    const int max_pass = A->max_pass > 0 ? A->max_pass : 64;
    double* vap[MCA_NG] = {X->q[ATJUP_S_H2O], X->q[ATJUP_S_NH3]};
    double* cld[MCA_NG] = {X->q[ATJUP_S_H2O_CLOUD], X->q[ATJUP_S_NH3_CLOUD]};
    double* ice[MCA_NG] = {X->q[ATJUP_S_H2O_ICE], X->q[ATJUP_S_NH3_ICE]};
    double* trf[MCA_NT] = {X->q[ATJUP_S_H2S], X->q[ATJUP_S_NH4SH]};
    int64_t st[8] = {0};
    mca_col* C = (mca_col*)malloc(sizeof(mca_col));
    if (!C || im > MCA_MAXI) { free(C); return; }
    for (int j = 0; j < jm; j++) {
        for (int k = 0; k < km; k++) {
            int i0 = 0;
            while (i0 < im && G->solid[IDX(i0, j, k)] == 1) i0++;
            int i1 = i0;
            while (i1 + 1 < im && G->solid[IDX(i1 + 1, j, k)] != 1) i1++;
            if (A->interior) { if (i0 == 0) i0 = 1; if (i1 == im - 1) i1 = im - 2; }
            if (i1 - i0 < 1) continue;
            memset(C->eq_ok, 0, sizeof C->eq_ok);
            memset(C->touched, 0, sizeof C->touched);
            int ok = 1;
            for (int i = i0; i <= i1 && ok; i++) {
                const size_t c = IDX(i, j, k);
                C->T[i] = C->T0[i] = S->t[c] * P->t_ref;
                C->p[i] = S->p_stat[c];
                C->z[i] = (double)X->layer_heights[i] * 1.0e3;
                double r = P->r_mix;
                if (P->local_rho) { const double rr = S->rho_mix[c]; r = (rr > 0.0 && isfinite(rr)) ? rr : P->r_mix; }
                C->rho[i] = r;
                if (!(C->T[i] > 0.0) || !(C->p[i] > 0.0) || !(C->rho[i] > 0.0) ||
                    !isfinite(C->T[i] + C->p[i] + C->rho[i]))
                    ok = 0;
            }
            if (!ok) { st[6]++; continue; }
            for (int i = i0; i <= i1 && ok; i++) {
                const size_t c = IDX(i, j, k);
                const double lo = (i > i0) ? 0.5 * (C->z[i - 1] + C->z[i]) : C->z[i0];
                const double hi = (i < i1) ? 0.5 * (C->z[i] + C->z[i + 1]) : C->z[i1];
                C->w[i] = C->rho[i] * (hi - lo);
                if (!(C->w[i] > 0.0)) ok = 0;
                double h = M.cp * C->T[i] + M.grav * C->z[i];
                for (int g = 0; g < MCA_NG; g++) {
                    const int x = i * MCA_NG + g;
                    C->qv[x] = dmax(0.0, vap[g][c]) / C->rho[i];
                    C->qc[x] = dmax(0.0, cld[g][c]) / C->rho[i];
                    C->qi[x] = dmax(0.0, ice[g][c]) / C->rho[i];
                    C->qt[x] = C->qv[x] + C->qc[x] + C->qi[x];
                    h -= M.g[g]->lv * C->qc[x] + M.g[g]->ls * C->qi[x];
                }
                for (int r = 0; r < MCA_NT; r++) {
                    C->qr[i * MCA_NT + r] = trf[r][c] / C->rho[i];
                    h -= M.tr_L[r] * C->qr[i * MCA_NT + r];
                }
                C->hL[i] = h;
            }
            if (!ok) { st[6]++; continue; }
            /* census of the unadjusted column */
            for (int i = i0; i < i1; i++) {
                int held = 0, moist = 0;
                const int u = mca_unstable(&M, C, i, i + 1, &held, &moist);
                C->cen_u[i] = (char)u;
                C->cen_m[i] = (char)moist;
                if (u || held) st[4]++;
                if (held) st[5]++;
            }
            memcpy(C->hL0, C->hL, sizeof C->hL);
            memcpy(C->qt0, C->qt, sizeof C->qt);
            memcpy(C->qr0, C->qr, sizeof C->qr);
            int passes = 0, changed = 1, fail = 0;
            int64_t layers = 0;
            while (changed && passes < max_pass && !fail) {
                changed = 0;
                passes++;
                int i = i0;
                while (i < i1 && !fail) {
                    int moist = 0, uns;
                    if (passes == 1 && !C->touched[i] && !C->touched[i + 1]) { uns = C->cen_u[i]; moist = C->cen_m[i]; }
                    else uns = mca_unstable(&M, C, i, i + 1, NULL, &moist);
                    if (!uns) { i++; continue; }
                    if (passes == 1) { if (moist) st[2]++; else st[3]++; }
                    int a = i, b = i + 1;
                    for (;;) {
                        if (!mca_mix(&M, C, a, b)) { fail = 1; break; }
                        int ext = 0;
                        if (a > i0 && mca_unstable(&M, C, a - 1, a, NULL, NULL)) { a--; ext = 1; }
                        if (b < i1 && mca_unstable(&M, C, b, b + 1, NULL, NULL)) { b++; ext = 1; }
                        if (!ext) break;
                    }
                    layers += b - a + 1;
                    changed = 1;
                    i = b;
                }
            }
            if (fail) { st[6]++; continue; }
            if (layers == 0) continue;
            if (relax < 1.0) {
                for (int q = i0; q <= i1 && !fail; q++) {
                    if (!C->touched[q]) continue;
                    C->hL[q] = C->hL0[q] + relax * (C->hL[q] - C->hL0[q]);
                    for (int g = 0; g < MCA_NG; g++) {
                        const int x = q * MCA_NG + g;
                        C->qt[x] = C->qt0[x] + relax * (C->qt[x] - C->qt0[x]);
                    }
                    for (int r = 0; r < MCA_NT; r++) {
                        const int x = q * MCA_NT + r;
                        C->qr[x] = C->qr0[x] + relax * (C->qr[x] - C->qr0[x]);
                    }
                    if (!mca_settle(&M, C, q)) fail = 1;
                }
                if (fail) { st[6]++; continue; }
            }
            for (int q = i0; q <= i1; q++) {
                if (!C->touched[q]) continue;
                const size_t c = IDX(q, j, k);
                S->t[c] = C->T[q] / P->t_ref;
                for (int g = 0; g < MCA_NG; g++) {
                    const int x = q * MCA_NG + g;
                    vap[g][c] = C->qv[x] * C->rho[q];
                    cld[g][c] = C->qc[x] * C->rho[q];
                    ice[g][c] = C->qi[x] * C->rho[q];
                }
                for (int r = 0; r < MCA_NT; r++) trf[r][c] = C->qr[q * MCA_NT + r] * C->rho[q];
            }
            st[0]++;
            st[1] += layers;
            if (passes > st[7]) st[7] = passes;
        }
    }
    free(C);
    if (stats) memcpy(stats, st, sizeof st);
}

void ora_iteration_phys(const AtjupParams* P, const AtjupPhysics* PH, const AtjupMicro* MC,
                        const AtjupMca* MCA, const ora_grid* G, ora_state* S, ora_phys* X,
                        int iter_n, int first, int sweeps) {
    const size_t N = (size_t)P->im * P->jm * P->km;
    if (iter_n % 2 == 0 || first) {
        ora_pressure_sweeps(P, G, S, sweeps, 1.0, NULL);
        ora_mixture_density(P, G, S);
        if (MC->radiation_on) ora_radiation(P, MC, G, S, X);
        if (MC->satadj_on) {
            const int sv[3] = {ATJUP_S_H2O, ATJUP_S_NH3, ATJUP_S_CH4};
            for (int q = 0; q < 3; q++)
                ora_satadj(P, G, &MC->gas[q], S->t, S->p_stat, S->rho_mix, X->q[sv[q]],
                           X->q[sv[q] + 1], X->q[sv[q] + 2], NULL);
        }
        if (MC->nh4sh_eq) ora_nh4sh_eq(P, MC, G, S, X);
        if (MC->precip_on) ora_precipitation(P, MC, G, S, X);
        /* ATJUP_RK_SCALAR_SYNC = 2 */
        const int sync[9] = {ATJUP_S_H2O, ATJUP_S_H2O_CLOUD, ATJUP_S_H2O_ICE, ATJUP_S_NH3,
                             ATJUP_S_NH3_CLOUD, ATJUP_S_NH3_ICE, ATJUP_S_CH4, ATJUP_S_CH4_CLOUD,
                             ATJUP_S_CH4_ICE};
        for (int q = 0; q < 9; q++) memcpy(X->qn[sync[q]], X->q[sync[q]], sizeof(double) * N);
        memcpy(S->tn, S->t, sizeof(double) * N);
        if (MC->nh4sh_eq) {
            memcpy(X->qn[ATJUP_S_H2S], X->q[ATJUP_S_H2S], sizeof(double) * N);
            memcpy(X->qn[ATJUP_S_NH4SH], X->q[ATJUP_S_NH4SH], sizeof(double) * N);
        }
        if (PH->turb_on) ora_turbulence(P, PH, G, S, X);
        ora_chemistry(P, MC, G, S, X);
    }
    ora_rk4_phys(P, PH, G, S, X);
    ora_bc_radius_x(P, G, S, X);
    ora_bc_theta_x(P, G, S, X);
    ora_bc_phi_x(P, G, S, X);
    ora_bc_solid_x(P, G, S, X);
    if (PH->turb_on) {                       /* ATJUP_TURB_WALL_HOLD 1 */
        ora_turb_wall_bc(P, PH, G, X);
        ora_turb_wall_omega(P, PH, G, X);
    }
    if (MCA && MCA->stride > 0 && iter_n % MCA->stride == 0) ora_mca(P, MC, MCA, G, S, X, NULL);
    if (P->shapiro_inloop > 0) {
        ora_shapiro(P, G, S->u, 4, P->shapiro_strength, P->shapiro_inloop, 1);
        ora_shapiro(P, G, S->v, 4, P->shapiro_strength, P->shapiro_inloop, 1);
        ora_shapiro(P, G, S->w, 4, P->shapiro_strength, P->shapiro_inloop, 1);
    }
    if (P->v_massbal_stride > 0 && iter_n % P->v_massbal_stride == 0) ora_balance_column_v(P, G, S);
    ora_clamp_species(P, X);
    ora_restore(P, S);
    for (int q = 0; q < ATJUP_S_COUNT; q++) memcpy(X->qn[q], X->q[q], sizeof(double) * N);
    memcpy(X->tken, X->tke, sizeof(double) * N);
    memcpy(X->disn, X->dis, sizeof(double) * N);
}


/* cJupiterModel::Forces (InitValues_Jup.cpp:742-812) and cJupiterModel::Latent_Heat
 * (Thermo_Jup.cpp:89-232): out[0..5] = CoriolisForce, CentrifugalForce, BuoyancyForce,
 * PresGradForce, Q_Latent, Q_Sensible. Forces fills i 1..im-2, j 1..jm-2, k 0..km-2 (the phi
 * ring); Latent_Heat zeroes its two fields at i = 0 and fills the same interior, i downwards.
 * Cells outside keep their values. coord_stretching is off (exp_rm = 1). */
static double ora_max(double a, double b) { return (a < b) ? b : a; }   /* std::max */

void ora_diagnostics(const AtjupParams* P, const AtjupMicro* MC, const ora_grid* G,
                     const double* t, const double* u, const double* v, const double* w,
                     const double* p_dyn, const double* p_stat, const double* h2o,
                     const double* nh3, double* const* out) {
    const int im = P->im, jm = P->jm, km = P->km;
    double *cor = out[0], *cen = out[1], *buo = out[2], *pgf = out[3], *ql = out[4], *qs = out[5];
    const double omega = P->omega;
    for (int i = 1; i < im - 1; i++)
        for (int j = 1; j < jm - 1; j++) {
            const double rm = G->rad[i];
            const double sinthe = sin(G->the[j]);
            double costhe = cos(G->the[j]);
            if (MC->costhe_abs && j > 90) costhe = -costhe;
            const double rmsinthe = rm * sinthe;
            for (int k = 0; k < km - 1; k++) {
                const int kw = phi_wrap(1, k - 1, km), ke = phi_wrap(1, k + 1, km);
                const size_t c = IDX(i, j, k);
                const double Cor_r = -2.0 * omega * sinthe * w[c];
                const double Cor_the = +2.0 * omega * costhe * w[c];
                const double Cor_phi = +2.0 * omega * (-costhe * v[c] + sinthe * u[c]);
                const double dpdr = (p_dyn[IDX(i + 1, j, k)] - p_dyn[IDX(i - 1, j, k)]) / (2.0 * P->dr);
                const double dpdthe = (p_dyn[IDX(i, j + 1, k)] - p_dyn[IDX(i, j - 1, k)]) / (2.0 * P->dthe);
                const double dpdphi = (p_dyn[IDX(i, j, ke)] - p_dyn[IDX(i, j, kw)]) / (2.0 * P->dphi);
                cor[c] = P->Coriolis * P->r_mix *
                         sqrt((pow(Cor_r, 2) + pow(Cor_the, 2) + pow(Cor_phi, 2)) / 3.0);
                cen[c] = P->centrifugal * P->r_mix * omega * omega * rm * (1.0 + fabs(sinthe));
                buo[c] = (t[c] > 0.0)
                             ? P->buoyancy * P->r_mix * P->g * (p_stat[c] + p_dyn[c] * P->p_dyn_to_bar) /
                                   (P->r_mix * P->R_mix * t[c] * P->t_ref) * 1e5
                             : 0.0;
                pgf[c] = -sqrt((pow(dpdr, 2) + pow(dpdthe / rm, 2) + pow(dpdphi / rmsinthe, 2)) / 3.0) *
                         P->p_dyn_to_bar * 1.0e5 / (P->L_atm * 1.0e3);
            }
        }
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) { ql[IDX(0, j, k)] = 0.0; qs[IDX(0, j, k)] = 0.0; }
    const double fix_lat = MC->qheat_scale ? (im - 1) / 1.0e3 : 1.0;
    const double fix_sen = MC->qheat_scale ? P->L_atm * (im - 1) * (im - 1) / 1.0e3 : 1.0;
    const AtjupGasParams *gw = &MC->gas[0], *ga = &MC->gas[1];
    for (int j = 1; j < jm - 1; j++) {
        const double sinthe = sin(G->the[j]);
        for (int k = 0; k < km - 1; k++) {
            const int kw = phi_wrap(1, k - 1, km), ke = phi_wrap(1, k + 1, km);
            for (int i = im - 2; i >= 1; i--) {
                const size_t c = IDX(i, j, k), cp = IDX(i + 1, j, k), cm = IDX(i - 1, j, k);
                const size_t cjp = IDX(i, j + 1, k), cjm = IDX(i, j - 1, k);
                const size_t ckp = IDX(i, j, ke), ckm = IDX(i, j, kw);
                const double rm = G->rad[i];
                const double rmsinthe = rm * sinthe;
                const double exp_rm = 1.0;
                double Latency_Ice = 0.0;
                const double t_u = t[c] * P->t_ref;
                const double p_u = p_stat[c];
                const double E_Rain = exp(MC->cc[0] / t_u + MC->cc[1]);
                const double E_Ice = exp(MC->cc[2] / t_u + MC->cc[3]);
                const double q_Rain = gw->ep * E_Rain / ora_max(p_u - E_Rain, 1.0e-12);
                const double q_Ice = gw->ep * E_Ice / ora_max(p_u - E_Ice, 1.0e-12);
                const double E_Rain_nh3 = exp(MC->cc[4] / t_u + MC->cc[5]);
                const double E_Ice_nh3 = exp(MC->cc[6] / t_u + MC->cc[7]);
                const double q_Rain_nh3 = ga->ep * E_Rain_nh3 / ora_max(p_u - E_Rain_nh3, 1.0e-12);
                const double q_Ice_nh3 = ga->ep * E_Ice_nh3 / ora_max(p_u - E_Ice_nh3, 1.0e-12);
                const double u_av = 0.5 * (u[cp] + u[cm]);
                const double v_av = 0.5 * (v[cp] + v[cm]);
                const double w_av = 0.5 * (w[cp] + w[cm]);
                const double velocity_av = -sqrt((pow(u_av, 2) + pow(v_av, 2) + pow(w_av, 2)) / 3.0);
                const double dtdr = (t[cp] - t[cm]) / (2.0 * P->dr) * exp_rm;
                const double dtdthe = (t[cjp] - t[cjm]) / (2.0 * rm * P->dthe);
                const double dtdphi = (t[ckp] - t[ckm]) / (2.0 * rmsinthe * P->dphi);
                const double dh2odr = (h2o[cp] - h2o[cm]) / (2.0 * P->dr) * exp_rm;
                const double dh2odthe = (h2o[cjp] - h2o[cjm]) / (2.0 * rm * P->dthe);
                const double dh2odphi = (h2o[ckp] - h2o[ckm]) / (2.0 * rmsinthe * P->dphi);
                const double dnh3dr = (nh3[cp] - nh3[cm]) / (2.0 * P->dr) * exp_rm;
                const double dnh3dthe = (nh3[cjp] - nh3[cjm]) / (2.0 * rm * P->dthe);
                const double dnh3dphi = (nh3[ckp] - nh3[ckm]) / (2.0 * rmsinthe * P->dphi);
                const double dtemp = dtdr + dtdthe + dtdphi;
                const double dh2o = dh2odr + dh2odthe + dh2odphi;
                const double dnh3 = dnh3dr + dnh3dthe + dnh3dphi;
                const double Lr = P->L_atm * (im - 1);
                if (h2o[c] >= q_Rain) ql[c] = gw->lv * velocity_av * dh2o * P->u_0 / Lr * fix_lat;
                else ql[c] = 0.0;
                if (h2o[c] >= q_Ice) Latency_Ice = gw->ls * velocity_av * dh2o * P->u_0 / Lr * fix_lat;
                else Latency_Ice = 0.0;
                if (nh3[c] >= q_Rain_nh3)
                    ql[c] = ql[c] + ga->lv * velocity_av * dnh3 * P->u_0 / Lr * fix_lat;
                if (nh3[c] >= q_Ice_nh3)
                    Latency_Ice = Latency_Ice + ga->ls * velocity_av * dnh3 * P->u_0 / Lr * fix_lat;
                ql[c] = ql[c] + Latency_Ice;
                qs[c] = P->r_mix * P->cp_mix * velocity_av * P->u_0 * dtemp * P->t_ref /
                        pow(P->L_atm * (im - 1), 2) * fix_sen;
                if (G->solid[c] == 1) { ql[c] = 0.0; qs[c] = 0.0; }
            }
        }
    }
}
