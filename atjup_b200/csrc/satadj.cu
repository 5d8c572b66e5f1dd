// Saturation adjustment of one condensable gas (SaturationAdjustment.h:255-746; Tao, Simpson and
// McCumber 1988, "An Ice-Water Saturation Adjustment").
//
// Every cell is independent, so the kernel is one thread per cell over the padded [i][j][KP]
// blocks, k fastest: a warp reads 32 consecutive doubles of each of t, p_stat, rho_mix and the
// gas's three species and writes t and the species back in place -- 10 streams of 8 bytes per
// cell, the whole of the kernel's HBM traffic. The per-cell work is a short FP64 iteration (at
// most 15 passes) around the Clausius-Clapeyron fit exp(C + (-L0/T + a ln T + b T)/(1e-3 R)),
// evaluated with CUDA's own exp and log. Expressions keep the reference's operand order and
// this file is compiled without FMA contraction, so the only departure from the reference is
// the last-bit rounding of exp and log.
//
// Lanes that skip (solid, dry, saturated) or converge early idle while the warp's slowest cell
// finishes; cells of one warp share i and j and differ only in longitude, so they tend to take
// the same branch.
#include "ctx.cuh"

namespace atjup {
namespace {

constexpr int SAT_PASSES = 15;          // iter_prec_end (SaturationAdjustment.h:250)
constexpr double SAT_Q_DIFF_MIN = 1.0e-3;  // q_diff_min (SaturationAdjustment.h:251)

// ATPhys::saturation_vapour_pressure (ATPhys.h:49-52) [bar]
__device__ __forceinline__ double svp(double T, double C, double L0, double R, double da,
                                      double db) {
    return exp(C + (-L0 / T + da * log(T) + db * T) / (1e-3 * R));
}

// Vapour target for q_c liquid and q_i ice at T from the liquid / ice saturation densities
// (SaturationAdjustment.h:513-520; the Newton probe at 564-571 makes the same choice).
__device__ __forceinline__ double target(const AtjupGasParams& g, double T, double qc, double qi,
                                         double ql, double qs, double tri) {
    if (qc > 0.0 && qi > 0.0) return (qc * ql + qi * qs) / (qc + qi);
    if (g.bergeron >= 2 && qc <= 0.0 && qi <= 0.0 && T < g.t_0) return qs;
    if (g.ice_entry && qc <= 0.0 && qi <= 0.0) {
        const double cn = T <= g.t_00 ? 0.0 : (T >= g.t_0 ? 1.0 : (T - g.t_00) * tri);
        return cn * ql + (1.0 - cn) * qs;
    }
    if (qi == 0.0) return ql;
    return qs;
}

struct SatArgs {
    double* t;
    const double* p_stat;
    const double* rho_mix;
    double *c, *cloud, *ice;
    const uint8_t* solid;
    unsigned long long* counters;   // adjusted, not converged, dry exits
    long long ncell_padded;
    int KP, km, local_rho;
    double t_ref, r_mix, cp_mix;
};

__global__ void __launch_bounds__(256) satadj_kernel(SatArgs a, AtjupGasParams g) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int adjusted = 0, noconv = 0, dryx = 0;
    if (q < a.ncell_padded && (int)(q % a.KP) < a.km) {
        double t_u = a.t[q] * a.t_ref;
        const double p_u = a.p_stat[q];
        double c = a.c[q], cl = a.cloud[q], ic = a.ice[q];
        const double c_in = c, cl_in = cl, ic_in = ic;
        bool t_dirty = false;
        double t_out = 0.0;
        const double tri = 1.0 / (g.t_0 - g.t_00);
        const double Lf = g.ls - g.lv;
        bool active = (t_u > 0.0) && (p_u > 0.0) && !a.solid[q];
        if (active) {
            double rho = a.r_mix;
            if (a.local_rho) {
                const double r = a.rho_mix[q];
                if (r > 0.0 && isfinite(r)) rho = r;
            }
            const double heat = a.cp_mix * rho;
            // entry bounds: melt above t_0, optional freeze below t_00, clip negatives
            if (t_u > g.t_0) {
                if (g.conserve) {
                    if (ic > 0.0) {
                        double dm = ic;
                        if (Lf > 0.0) {
                            const double cap = heat * (t_u - g.t_0) / Lf;
                            if (dm > cap) dm = cap;
                            t_u -= Lf * dm / heat;
                            t_out = t_u / a.t_ref;
                            t_dirty = true;
                        }
                        ic -= dm;
                        cl += dm;
                    }
                } else {
                    ic = 0.0;
                }
            }
            if (g.freeze && g.conserve && g.t_00 > 0.0 && g.t_00 < g.t_0 && t_u < g.t_00 &&
                cl > 0.0) {
                double dm = cl;
                if (Lf > 0.0) {
                    const double cap = heat * (g.t_00 - t_u) / Lf;
                    if (dm > cap) dm = cap;
                    t_u += Lf * dm / heat;
                    t_out = t_u / a.t_ref;
                    t_dirty = true;
                }
                cl -= dm;
                ic += dm;
            }
            if (c < 0.0) c = 0.0;
            if (cl < 0.0) cl = 0.0;
            if (ic < 0.0) ic = 0.0;

            // entry test (SaturationAdjustment.h:422-452); every saturation density is
            // ((rho * ep) * E) / p_u, the reference's rho_c * ep * E / p_u
            const double rep = rho * g.ep;
            const double q_rain0 = rep * svp(t_u, g.C, g.L0, g.R, g.del_alf, g.del_bet) / p_u;
            bool enter = q_rain0 > 0.0;
            if (enter) {
                double q_entry = q_rain0;
                if (g.ice_entry && cl <= 0.0 && ic <= 0.0) {
                    const double cnd0 = t_u <= g.t_00 ? 0.0
                                      : (t_u >= g.t_0 ? 1.0 : (t_u - g.t_00) * tri);
                    if (cnd0 < 1.0)
                        q_entry = cnd0 * q_rain0 + (1.0 - cnd0) * rho * g.ep
                                * svp(t_u, g.C_i, g.L0_i, g.R, g.del_alf_i, g.del_bet_i) / p_u;
                }
                if (g.bergeron >= 2 && cl <= 0.0 && ic <= 0.0 && t_u < g.t_0)
                    q_entry = rep * svp(t_u, g.C_i, g.L0_i, g.R, g.del_alf_i, g.del_bet_i) / p_u;
                if (c <= q_entry) {
                    if (!g.evap || !g.conserve || (cl <= 0.0 && ic <= 0.0)) {
                        enter = false;
                    } else {
                        const double q_ice0 =
                            rep * svp(t_u, g.C_i, g.L0_i, g.R, g.del_alf_i, g.del_bet_i) / p_u;
                        double q_t0;
                        if (cl > 0.0 && ic > 0.0) q_t0 = (cl * q_rain0 + ic * q_ice0) / (cl + ic);
                        else if (ic <= 0.0) q_t0 = q_rain0;
                        else q_t0 = q_ice0;
                        if (fabs(c - q_t0) <= SAT_Q_DIFF_MIN * q_t0) enter = false;
                    }
                }
            }

            if (enter) {
                // mixed-phase iteration (SaturationAdjustment.h:454-604)
                double qv = c, qc = cl, qi = ic, T = t_u, hyp = qv, q_rain_now = q_rain0;
                bool found = false, dry = false;
                for (int itr = 1; itr <= SAT_PASSES; itr++) {
                    double CND = (T - g.t_00) * tri;
                    double DEP = (g.t_0 - T) * tri;
                    if (T <= g.t_00) { CND = 0.0; DEP = 1.0; }
                    if (T >= g.t_0) { CND = 1.0; DEP = 0.0; }
                    const bool berg = g.bergeron != 0 && T < g.t_0 && qv <= q_rain_now &&
                                      (qi > 0.0 || (g.bergeron >= 2 && qc <= 0.0));
                    if (berg) {
                        CND = 0.0;
                        DEP = 1.0;
                        if (qc > 0.0) {
                            T -= g.lv * qc / heat;
                            qv += qc;
                            qc = 0.0;
                        }
                    }
                    double dv = hyp - qv;
                    double dc = -dv * CND;
                    double di = -dv * DEP;
                    if (g.conserve) {
                        if (dv < -qv) { dv = -qv; dc = -dv * CND; di = -dv * DEP; }
                        if (qc + dc < 0.0) { const double ex = -(qc + dc); dc = -qc; di -= ex; }
                        if (qi + di < 0.0) {
                            const double ex = -(qi + di);
                            di = -qi;
                            dc -= ex;
                            if (qc + dc < 0.0) dc = -qc;
                        }
                        dv = -(dc + di);
                    }
                    T += (g.lv * dc + g.ls * di) / heat;
                    qv += dv;
                    qc += dc;
                    qi += di;
                    if (qv < 0.0) qv = 0.0;
                    if (qc < 0.0) qc = 0.0;
                    if (qi < 0.0) qi = 0.0;

                    const double ql = rep * svp(T, g.C, g.L0, g.R, g.del_alf, g.del_bet) / p_u;
                    const double qs =
                        rep * svp(T, g.C_i, g.L0_i, g.R, g.del_alf_i, g.del_bet_i) / p_u;
                    q_rain_now = ql;
                    hyp = target(g, T, qc, qi, ql, qs, tri);

                    if (T >= g.t_0) {
                        if (g.conserve) {
                            if (qi > 0.0) {
                                double dm = qi;
                                if (Lf > 0.0) {
                                    const double cap = heat * (T - g.t_0) / Lf;
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
                    if (q_diff <= SAT_Q_DIFF_MIN) { found = true; break; }
                    if (g.dry_exit && g.conserve && qc <= 0.0 && qi <= 0.0 && qv < hyp) {
                        dry = true;
                        break;
                    }
                    if (g.newton) {
                        const double dT = 0.1;
                        const double qld =
                            rep * svp(T + dT, g.C, g.L0, g.R, g.del_alf, g.del_bet) / p_u;
                        const double qsd =
                            rep * svp(T + dT, g.C_i, g.L0_i, g.R, g.del_alf_i, g.del_bet_i) / p_u;
                        const double hyp_d = target(g, T, qc, qi, qld, qsd, tri);
                        double CNDn = (T - g.t_00) * tri;
                        if (T <= g.t_00) CNDn = 0.0;
                        if (T >= g.t_0) CNDn = 1.0;
                        if (berg) CNDn = 0.0;
                        const double G = (g.lv * CNDn + g.ls * (1.0 - CNDn)) / heat *
                                         (hyp_d - hyp) / dT;
                        double w = 1.0 / (1.0 + (G < 0.0 ? 0.0 : G));
                        if (w < 0.05) w = 0.05;
                        hyp = qv + w * (hyp - qv);
                    } else {
                        hyp = 0.5 * (hyp + qv);
                    }
                }
                adjusted = 1;
                noconv = (!found && !dry) ? 1 : 0;
                dryx = dry ? 1 : 0;
                c = qv;
                cl = qc;
                ic = qi;
                t_out = T / a.t_ref;
                t_dirty = true;
            }
        }
        // final clamp (SaturationAdjustment.h:673-685) applies to every cell, solid included
        if (c <= 0.0) c = 0.0;
        if (cl <= 0.0) cl = 0.0;
        if (ic <= 0.0) ic = 0.0;
        if (t_dirty) a.t[q] = t_out;
        // write only what changed: a skipped cell whose species were already >= 0 costs no store
        if (__double_as_longlong(c) != __double_as_longlong(c_in)) a.c[q] = c;
        if (__double_as_longlong(cl) != __double_as_longlong(cl_in)) a.cloud[q] = cl;
        if (__double_as_longlong(ic) != __double_as_longlong(ic_in)) a.ice[q] = ic;
    }
    // event counts: warp sums, one atomic per warp and counter
    const unsigned full = 0xffffffffu;
    const int sa = __reduce_add_sync(full, adjusted);
    const int sn = __reduce_add_sync(full, noconv);
    const int sd = __reduce_add_sync(full, dryx);
    if ((threadIdx.x & 31) == 0) {
        if (sa) atomicAdd(&a.counters[0], (unsigned long long)sa);
        if (sn) atomicAdd(&a.counters[1], (unsigned long long)sn);
        if (sd) atomicAdd(&a.counters[2], (unsigned long long)sd);
    }
}

}  // namespace

int launch_satadj(AtjupCtx* c, int gas, const AtjupGasParams& gp) {
    static const int ids[3][3] = {{ATJUP_F_H2O, ATJUP_F_H2O_CLOUD, ATJUP_F_H2O_ICE},
                                  {ATJUP_F_NH3, ATJUP_F_NH3_CLOUD, ATJUP_F_NH3_ICE},
                                  {ATJUP_F_CH4, ATJUP_F_CH4_CLOUD, ATJUP_F_CH4_ICE}};
    SatArgs a;
    a.t = c->f[ATJUP_F_T];
    a.p_stat = c->f[ATJUP_F_P_STAT];
    a.rho_mix = c->f[ATJUP_F_RHO_MIX];
    a.c = c->f[ids[gas][0]];
    a.cloud = c->f[ids[gas][1]];
    a.ice = c->f[ids[gas][2]];
    a.solid = c->solid;
    a.counters = c->counters;
    a.ncell_padded = (long long)c->NP;
    a.KP = c->KP;
    a.km = c->P.km;
    a.local_rho = c->P.local_rho;
    a.t_ref = c->P.t_ref;
    a.r_mix = c->P.r_mix;
    a.cp_mix = c->P.cp_mix;
    ATJUP_CUDA(cudaMemsetAsync(c->counters, 0, 8 * sizeof(unsigned long long), c->stream));
    const int threads = 256;
    const long long blocks = ((long long)c->NP + threads - 1) / threads;
    satadj_kernel<<<(unsigned)blocks, threads, 0, c->stream>>>(a, gp);
    c->launches++;
    ATJUP_CHECK_LAUNCH("satadj_kernel");
    return ATJUP_OK;
}

}  // namespace atjup
